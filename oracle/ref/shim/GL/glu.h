/* Header shim: see GL/gl.h. */
#ifndef ENC_ORACLE_SHIM_GLU_H
#define ENC_ORACLE_SHIM_GLU_H
#include "GL/gl.h"
static inline const GLubyte* gluErrorString(GLenum) { return (const GLubyte*)""; }
static inline void gluPerspective(double, double, double, double) {}
#endif
