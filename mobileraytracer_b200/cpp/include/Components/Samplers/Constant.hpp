// Constant.hpp - same path as the reference header (app/Components/Samplers/Constant.hpp); the classes live in b200_api.hpp.
#pragma once
#include "MobileRT/b200_api.hpp"
