// Stand-in for oomph::message_buffer (test infrastructure): an owning byte buffer, or a view of
// caller-provided memory.
#pragma once

#include <cstddef>
#include <memory>
#include <vector>

namespace oomph
{
template<typename T>
class message_buffer
{
    std::shared_ptr<std::vector<T>> m_own;
    T* m_ptr = nullptr;
    std::size_t m_size = 0;

  public:
    message_buffer() = default;
    explicit message_buffer(std::size_t n)
    : m_own(std::make_shared<std::vector<T>>(n))
    , m_ptr(m_own->data())
    , m_size(n)
    {
    }
    message_buffer(T* ptr, std::size_t n)
    : m_ptr(ptr)
    , m_size(n)
    {
    }
    T* data() noexcept { return m_ptr; }
    const T* data() const noexcept { return m_ptr; }
    std::size_t size() const noexcept { return m_size; }
    explicit operator bool() const noexcept { return m_ptr != nullptr; }
    bool on_device() const noexcept { return false; }
    T* device_data() noexcept { return nullptr; }
    int device_id() const noexcept { return 0; }
};
} // namespace oomph
