/* Included first into the reference sources built under oracle/_ref: the
 * standard headers that the shims (included by the reference inside its own
 * namespace) rely on, and the build revision string the reference prints.
 * TEST INFRASTRUCTURE ONLY. */
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#ifndef XAMG_REVISION
#define XAMG_REVISION "reference sources built against single-process shims"
#endif
