// OBJLoader.hpp - same path as the reference header (app/Components/ObjectLoaders/OBJLoader.hpp); the class lives in b200_api.hpp.
#pragma once
#include "MobileRT/b200_api.hpp"
