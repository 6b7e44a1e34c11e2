// Stand-in for oomph::communicator (test infrastructure): a loopback transport for one rank.
// recv() posts a buffer with its completion callback; send() copies the message into the posted
// buffer with the same tag (as an MPI self-send copies it) or keeps it until such a receive is
// posted; progress()/wait_all() run the callbacks of the completed receives.
#pragma once

#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <vector>

#include <oomph/message_buffer.hpp>

namespace oomph
{
using rank_type = int;
using tag_type = int;

class send_request
{
  public:
    bool is_ready() const noexcept { return true; }
    bool test() const noexcept { return true; }
    void wait() const noexcept {}
};

class recv_request
{
  public:
    bool is_ready() const noexcept { return true; }
    bool test() const noexcept { return true; }
    void wait() const noexcept {}
};

class communicator
{
  public:
    struct state;

  private:
    struct posted
    {
        unsigned char* buf;
        std::size_t size;
        tag_type tag;
        bool filled;
        std::function<void()> done;
    };
    struct unexpected
    {
        tag_type tag;
        std::vector<unsigned char> data;
    };
  public:
    struct state
    {
        std::vector<posted> recvs;
        std::vector<unexpected> early;
    };

  private:
    std::shared_ptr<state> m_state = std::make_shared<state>();

  public:
    communicator() = default;
    // communicators of one context share the process's mailbox, as MPI communicators built on
    // one MPI communicator match each other's messages
    explicit communicator(std::shared_ptr<state> s)
    : m_state(std::move(s))
    {
    }

    rank_type rank() const noexcept { return 0; }
    rank_type size() const noexcept { return 1; }

    template<typename T>
    message_buffer<T> make_buffer(std::size_t n)
    {
        return message_buffer<T>(n);
    }
    template<typename T>
    message_buffer<T> make_buffer(T* ptr, std::size_t n)
    {
        return message_buffer<T>(ptr, n);
    }

    template<typename T, typename Callback>
    recv_request recv(message_buffer<T>& m, rank_type src, tag_type tag, Callback&& cb)
    {
        auto* msg = &m;
        posted p{reinterpret_cast<unsigned char*>(m.data()), m.size() * sizeof(T), tag, false,
            [msg, src, tag, cb]() mutable { cb(*msg, src, tag); }};
        for (auto it = m_state->early.begin(); it != m_state->early.end(); ++it)
            if (it->tag == tag)
            {
                std::memcpy(p.buf, it->data.data(), std::min(p.size, it->data.size()));
                p.filled = true;
                m_state->early.erase(it);
                break;
            }
        m_state->recvs.push_back(std::move(p));
        return {};
    }

    template<typename T>
    send_request send(message_buffer<T>& m, rank_type, tag_type tag)
    {
        const auto* bytes = reinterpret_cast<const unsigned char*>(m.data());
        const std::size_t n = m.size() * sizeof(T);
        for (auto& p : m_state->recvs)
            if (!p.filled && p.tag == tag)
            {
                std::memcpy(p.buf, bytes, std::min(p.size, n));
                p.filled = true;
                return {};
            }
        m_state->early.push_back(unexpected{tag, std::vector<unsigned char>(bytes, bytes + n)});
        return {};
    }

    // send with a completion callback (the in-place receive's sends): the copy is done at once
    template<typename T, typename Callback>
    send_request send(message_buffer<T>& m, rank_type dst, tag_type tag, Callback&& cb)
    {
        send(m, dst, tag);
        cb(m, dst, tag);
        return {};
    }

    void progress()
    {
        auto& r = m_state->recvs;
        for (std::size_t i = 0; i < r.size();)
        {
            if (r[i].filled)
            {
                auto done = std::move(r[i].done);
                r.erase(r.begin() + i);
                done();
            }
            else
                ++i;
        }
    }

    bool is_ready() const noexcept { return m_state->recvs.empty(); }

    void wait_all()
    {
        progress();
        if (!m_state->recvs.empty())
            throw std::runtime_error("loopback transport: a posted receive has no matching send");
    }
};
} // namespace oomph
