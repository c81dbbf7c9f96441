// Adjacency-text loader (declarations also in include/dmolp_b200.h).
#pragma once
#include "../../include/dmolp_b200.h"
