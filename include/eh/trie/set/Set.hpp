// Set.hpp -- the reference header of that name, provided by the B200 layer.
#pragma once
#include "../../eh_dropin.hpp"
