/* Stand-in for the precompiled header the reference's SphBase.h includes
 * (SphBase.h:29).  It pulls in the glm stand-in.  Test infrastructure only. */
#ifndef ORACLE_STDAFX_SHIM_H_
#define ORACLE_STDAFX_SHIM_H_
#include <cstdio>
#include <cmath>
#include "glm_shim.h"
#endif
