// Host-side icosahedral grid builder of thorx; the C declarations are in include/thorx.h.
#pragma once
#include "../../include/thorx.h"
