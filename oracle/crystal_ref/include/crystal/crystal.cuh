// Test infrastructure: lets the reference's Crystal programs, which include
// "crystal/crystal.cuh", compile against this repository's Crystal API header instead.
#pragma once
#include "crystal_b200.cuh"
