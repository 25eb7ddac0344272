// Test infrastructure (oracle): see optix.h in this directory.
#pragma once
#include "optix.h"
