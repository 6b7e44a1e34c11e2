// Stand-in for hwmalloc's device helpers (test infrastructure): no device.
#pragma once

#include <cstddef>
#include <cstdlib>
#include <cstring>

namespace hwmalloc
{
inline int get_num_devices() { return 0; }
inline int get_device_id() { return 0; }
inline void set_device_id(int) {}
inline void* device_malloc(std::size_t n) { return std::malloc(n); }
inline void device_free(void* p) { std::free(p); }
inline void memcpy_to_device(void* dst, const void* src, std::size_t n) { std::memcpy(dst, src, n); }
inline void memcpy_to_host(void* dst, const void* src, std::size_t n) { std::memcpy(dst, src, n); }
} // namespace hwmalloc
