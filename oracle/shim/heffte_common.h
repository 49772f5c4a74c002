/* TEST INFRASTRUCTURE ONLY: see heffte.h. */
#ifndef ORC_SHIM_HEFFTE_COMMON_H
#define ORC_SHIM_HEFFTE_COMMON_H
#include "heffte.h"
#endif
