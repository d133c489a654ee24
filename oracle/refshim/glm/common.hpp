// Project-written GLM API shim entry header (see shim_core.hpp).
#pragma once
#include "shim_core.hpp"
