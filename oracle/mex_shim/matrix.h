/* Part of the MEX stand-in (see mex.h in this folder). */
#pragma once
#include "mex.h"
