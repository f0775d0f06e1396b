// Force-included ahead of every reference translation unit in the oracle build.
// TEST INFRASTRUCTURE ONLY.  The reference's force.hpp/energy.hpp include
// rendering/RenderEngine.hpp, which the oracle build stubs out by predefining
// its include guard (the renderer needs WebGPU/ImGui, absent here); that header
// also supplied these standard headers transitively.
#pragma once
#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <math.h>
#include <iostream>
#include <memory>
#include <string>
#include <vector>
