// Status codes shared by the host and device sources.
#pragma once

#include "../../include/b200_nufft.h"
