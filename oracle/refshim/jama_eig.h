/* Stand-in for JAMA's eigen header (surface_field.h:11); surface_field.cpp
 * uses only the SVD (jama_svd.h).  Test infrastructure only. */
#ifndef REFSHIM_JAMA_EIG_H_
#define REFSHIM_JAMA_EIG_H_
#include "jama_svd.h"
#endif
