// Stand-in for gridtools::array (test infrastructure): a fixed-size aggregate array.
#pragma once

#include <cstddef>

#ifndef GT_FUNCTION
#define GT_FUNCTION
#endif

namespace gridtools
{
template<typename T, std::size_t N>
struct array
{
    T m_data[N];

    using value_type = T;
    using iterator = T*;
    using const_iterator = const T*;

    static constexpr std::size_t size() noexcept { return N; }
    constexpr T& operator[](std::size_t i) noexcept { return m_data[i]; }
    constexpr const T& operator[](std::size_t i) const noexcept { return m_data[i]; }
    T* begin() noexcept { return m_data; }
    T* end() noexcept { return m_data + N; }
    const T* begin() const noexcept { return m_data; }
    const T* end() const noexcept { return m_data + N; }
    T* data() noexcept { return m_data; }
    const T* data() const noexcept { return m_data; }
};
} // namespace gridtools
