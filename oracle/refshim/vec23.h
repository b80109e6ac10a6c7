/* surface_field.h includes "vec23.h"; the reference's file is Vec23.h
 * (case-sensitive file systems).  Test infrastructure only. */
#include "Vec23.h"
