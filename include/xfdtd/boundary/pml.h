// xfdtd/boundary/pml.h: the include path reference programs use for this part of the API.
// This library declares its whole C++ API in xfdtd/xfdtd.h.
#pragma once
#include "../xfdtd.h"
