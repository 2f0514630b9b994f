/*
 * Test infrastructure (oracle build only): pre-included before every
 * reference translation unit.  The reference relies on transitive standard
 * includes that modern libstdc++ no longer provides, and defines a global
 * `log2(float)` (reference utils/utils.hpp:289) that clashes with <cmath>;
 * the macro renames the reference's function inside the oracle build.
 */
#include <cmath>
#include <math.h>
#include <algorithm>
#include <array>
#include <vector>
#include <iomanip>
#include <thread>
#include <string>
#include <cstring>
#include <limits>
#define log2 psy_log2
