// See tbb.h: the shim defines parallel_for there.
#pragma once
#include "tbb.h"
