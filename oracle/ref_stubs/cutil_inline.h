/* Stand-in for the SDK cutil_inline header: forwards to the cutil stand-in. */
#pragma once
#include "cutil.h"
