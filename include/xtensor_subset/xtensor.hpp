// xtensor-compatible umbrella include: the subset lives in xtensor/xt_core.hpp.
#pragma once
#include "xtensor/xt_core.hpp"
