// TEST INFRASTRUCTURE ONLY: see tbb.h in this folder.
#include "tbb.h"
