// hhs_internal.h -- shared declarations of the library's translation units.
#pragma once
#include "../../include/hhs.h"
