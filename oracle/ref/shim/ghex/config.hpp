// GHEX's build-generated configuration header, written for a CPU-only build (test
// infrastructure): no GPU, no RMA, the exchange schedule of communication_object.hpp.
#pragma once

#include <oomph/config.hpp>
#include <tuple>

#define GHEX_VERSION 40
#define GHEX_VERSION_MAJOR 0
#define GHEX_VERSION_MINOR 4
#define GHEX_VERSION_PATCH 0
#define GHEX_NO_RMA
#define GHEX_GPU_MODE none
#define GHEX_DEVICE_NONE

namespace ghex
{
struct cpu
{
};
struct gpu
{
};
using arch_list = std::tuple<cpu>;
} // namespace ghex
