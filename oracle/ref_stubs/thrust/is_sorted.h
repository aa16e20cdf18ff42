/* thrust/is_sorted.h no longer exists as a separate header; is_sorted lives in thrust/sort.h. */
#pragma once
#include <thrust/sort.h>
