/*
 * Forced-include header used only when compiling the upstream CICY_geom
 * sources into the test oracle (oracle/_ref).  It is test infrastructure,
 * never part of the shipped library.
 *
 * Upstream Hns.h declares foutstream::operator<< for both `size_t` and
 * `unsigned long` (Hns.h:50,52); on LP64 Linux those are the same type and
 * g++ rejects the redeclaration.  Instead of patching a copy of the sources,
 * every standard header the upstream code uses is included first (so their
 * include guards are closed) and `size_t` is then re-spelled as a distinct
 * 64-bit unsigned type for the upstream translation units only.  No
 * arithmetic changes: both types are 64-bit unsigned.
 */
#ifndef CICY_REF_COMPAT_H
#define CICY_REF_COMPAT_H
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <map>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <vector>
#include <stdlib.h>
#include <time.h>
typedef unsigned long long cicy_ref_size_t;
#define size_t cicy_ref_size_t
#endif
