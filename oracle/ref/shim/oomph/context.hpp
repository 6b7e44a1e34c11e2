// Stand-in for oomph::context (test infrastructure).
#pragma once

#include <mpi.h>

#include <oomph/communicator.hpp>
#include <oomph/message_buffer.hpp>

namespace oomph
{
class context
{
    MPI_Comm m_comm;
    std::shared_ptr<communicator::state> m_mailbox = std::make_shared<communicator::state>();

  public:
    context(MPI_Comm comm, bool /*thread_safe*/ = true)
    : m_comm(comm)
    {
    }
    MPI_Comm mpi_comm() const noexcept { return m_comm; }
    communicator get_communicator() { return communicator{m_mailbox}; }
    template<typename T>
    message_buffer<T> make_buffer(std::size_t n)
    {
        return message_buffer<T>(n);
    }
};
} // namespace oomph
