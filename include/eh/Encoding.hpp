// Encoding.hpp -- the reference header of that name, provided by the B200 layer (eh_dropin.hpp).
#pragma once
#include "eh_dropin.hpp"
