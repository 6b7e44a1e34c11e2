// Stand-in for gridtools::layout_map (test infrastructure): per dimension the position in the
// storage order (the largest value has stride 1).
#pragma once

#include <cstddef>

namespace gridtools
{
template<int... Args>
struct layout_map
{
    static constexpr std::size_t length = sizeof...(Args);
    static constexpr std::size_t masked_length = ((Args >= 0 ? 1 : 0) + ... + 0);
    static constexpr int at(int i)
    {
        constexpr int v[] = {Args...};
        return v[i];
    }
    static constexpr int find(int value)
    {
        constexpr int v[] = {Args...};
        for (std::size_t i = 0; i < length; ++i)
            if (v[i] == value) return (int)i;
        return -1;
    }
};
} // namespace gridtools
