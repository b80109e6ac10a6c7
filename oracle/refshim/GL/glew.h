/* No-op stand-in for GL/glew.h, included by the reference's PciSph.cpp:21
 * (its particle-drawing routine, PciSph.cpp:509-524, calls these).  The
 * oracle never draws, so the calls do nothing.  Test infrastructure only. */
#ifndef ORACLE_GLEW_SHIM_H_
#define ORACLE_GLEW_SHIM_H_
#define GL_FRONT_AND_BACK 0
#define GL_AMBIENT_AND_DIFFUSE 0
inline void glMaterialfv(int, int, const float*) {}
inline void glPushMatrix() {}
inline void glPopMatrix() {}
inline void glTranslatef(float, float, float) {}
#endif
