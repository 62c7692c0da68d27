// xtensor-compatible include path: the subset lives in xt_core.hpp.
#pragma once
#include "xt_core.hpp"
