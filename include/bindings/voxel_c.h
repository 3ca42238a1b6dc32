/* Forwarding header: lets callers written against the reference's
 * "bindings/voxel_c.h" include path (the Go cgo preamble, examples/c_test.cpp)
 * compile unchanged with -I <repo>/include. */
#pragma once
#include "../voxel_c.h"
