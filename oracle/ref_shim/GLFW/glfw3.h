// Empty stand-in: the reference octree files include GLFW but call nothing from it.
#pragma once
