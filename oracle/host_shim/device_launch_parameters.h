// TEST INFRASTRUCTURE ONLY: host stand-in (see cuda_runtime.h in this folder).
#pragma once
#include "cuda_runtime.h"
