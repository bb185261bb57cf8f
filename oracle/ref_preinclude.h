/*
 * ref_preinclude.h — test infrastructure, not product code.
 * Force-included (-include) before every reference translation unit of the
 * oracle/_ref builds: the standard headers are pulled in first, then access
 * specifiers are widened so that ref_harness.cpp can snapshot the reference's
 * internal state. No reference source is modified and code generation is
 * unchanged (access control does not affect layout or codegen in GCC).
 */
#include <algorithm>
#include <atomic>
#include <cassert>
#include <chrono>
#include <ciso646>
#include <cmath>
#include <complex>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <omp.h>
#include <random>
#include <set>
#include <sstream>
#include <stack>
#include <stdexcept>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>
#define private public
#define protected public
