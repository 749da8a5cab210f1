// Common prelude for the translation units that compile the reference's own
// kernel files in place (they are #included from the reference tree, never
// copied). TEST INFRASTRUCTURE ONLY: the resulting oracle/_ref/*.so files are
// checkers for the CUDA path and the timed CPU reference arm.
#pragma once
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <type_traits>

#include "arm_sme.h"
#include "arm_sve.h"

#define SKREF_EXPORT extern "C" __attribute__((visibility("default")))
