// output.h stand-in (TEST INFRASTRUCTURE, see qshim.h): no output files.
#pragma once
#include "qshim.h"
