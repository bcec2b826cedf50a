// TEST INFRASTRUCTURE ONLY: host stand-in (see thrust_host.h).
#pragma once
#include "thrust_host.h"
