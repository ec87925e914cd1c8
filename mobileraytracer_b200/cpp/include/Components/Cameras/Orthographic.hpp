// Orthographic.hpp - same path as the reference header (app/Components/Cameras/Orthographic.hpp); the classes live in b200_api.hpp.
#pragma once
#include "MobileRT/b200_api.hpp"
