/* Test infrastructure only (oracle build). The reference's SphericalHarmonics.cc
 * includes <legendre_rule.hpp>; the reference tree ships legendre_rule.h, whose
 * declarations use std::string without including <string>. */
#include <string>
#include "legendre_rule.h"
