/*
 * ref_shim.h — force-included (g++ -include) into every translation unit of
 * the reference-CPU harness build.  It only redirects the reference's printf
 * calls to ppm_ref_printf (defined in ref_harness.cpp), which counts the
 * out-of-range messages of cpu/hunt.hpp:16-18,104,111 instead of printing
 * them (tens of millions of lines on some workloads) and forwards everything
 * else to stderr.  The reference sources themselves are compiled unchanged.
 * TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <numeric>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

extern "C" int ppm_ref_printf(const char* fmt, ...);
namespace std {
using ::ppm_ref_printf;
}
#define printf ppm_ref_printf
