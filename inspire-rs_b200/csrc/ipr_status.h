// ipr_status.h — status codes shared by the product sources (public values in include/ipr_b200.h)
#pragma once
#include "ipr_b200.h"
