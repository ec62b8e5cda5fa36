// Forwards to the project-written glm subset (test infrastructure).
#pragma once
#include "vec3.hpp"
