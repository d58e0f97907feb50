// Test infrastructure: stand-in for GLM's umbrella header (only vec3 is used).
#pragma once
#include "vec3.hpp"
