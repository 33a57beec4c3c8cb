// Test infrastructure only (oracle): the ray/hit types live in rtcore.h of this shim.
#pragma once
#include "rtcore.h"
