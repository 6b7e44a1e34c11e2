// Stand-in for oomph::barrier (test infrastructure): a single rank needs none.
#pragma once
#include <oomph/context.hpp>
