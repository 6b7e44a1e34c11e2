// Field memory shared between processes (CUDA IPC), for the sharded exchange: every process maps
// the fields of the other processes' domains into its own address space, and one exchange kernel
// per process moves its part of the halos directly between the GPUs' memories (peer loads and
// stores over NVLink), with no message buffers.
#pragma once

#include <cstdint>

namespace ghexb
{
constexpr int k_ipc_handle_bytes = 64;

// The IPC handle of the device allocation holding `ptr` and the byte offset of `ptr` in it.
void ipc_export(const void* ptr, unsigned char* handle, int64_t* offset);
// Maps the allocation of `handle` (exported by another process) into this one, once per handle
// however often it is opened; returns the mapped address of byte `offset`.
void* ipc_open(const unsigned char* handle, int64_t offset);
// Drops one opening of `handle`; the mapping is released with the last one.
void ipc_close(const unsigned char* handle);
} // namespace ghexb
