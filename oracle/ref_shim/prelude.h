/* Forced prelude for compiling the reference's CPU sources (test infrastructure).
 *
 * The reference defines function-like min/max macros (src/sim/es/device_macros.h:42-43
 * and the Win32 header), which break the standard library headers if those are
 * included afterwards. Pulling every standard header the reference uses in first
 * makes the later includes no-ops.
 */
#pragma once
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <clocale>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
using std::abs;
