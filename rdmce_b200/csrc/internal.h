// internal.h -- declarations shared by the engine's translation units.
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/rdmce.h"
