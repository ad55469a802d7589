// Force-included header that stands in for the reference's
// single_gpu_sph_src/header/std_header.cuh:1-31 when the reference's own
// hot-path kernels are compiled for the checker library oracle/_ref.  The
// original header pulls in VTK and nlohmann/json, neither of which the
// compiled files (hash.cu, sort.cu, delta_ns.cu, time_int.cu, init.cu,
// check.cu) use; this shim provides the standard and Thrust headers they do
// use.  Test infrastructure only.
#pragma once
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/extrema.h>
#include <thrust/sort.h>
