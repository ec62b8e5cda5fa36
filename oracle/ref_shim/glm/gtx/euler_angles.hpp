// Empty: the reference octree files include this header but use nothing from it.
#pragma once
#include "../vec3.hpp"
