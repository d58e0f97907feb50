// Test infrastructure: empty stand-in; the reference includes this header without using it.
#pragma once
#include "vec3.hpp"
