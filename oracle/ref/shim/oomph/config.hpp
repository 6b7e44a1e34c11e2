// Stand-in for the oomph transport's configuration header (test infrastructure): CPU only, no
// barrier.
#pragma once
#define OOMPH_DEVICE_NONE
#define OOMPH_ENABLE_BARRIER 0
