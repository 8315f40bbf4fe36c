/* Header shim: GL scalar types and inert stand-ins for the few GL calls the
 * reference's model/AABB/camera helpers name.  None of them runs on the query
 * path (closest hit, kd-tree / BVH build, photon map, the camera basis);
 * they exist only so the reference's own .cpp files compile unmodified
 * without a graphics stack. */
#ifndef ENC_ORACLE_SHIM_GL_H
#define ENC_ORACLE_SHIM_GL_H
typedef unsigned int GLuint;
typedef unsigned int GLenum;
typedef int GLint;
typedef float GLfloat;
typedef unsigned char GLubyte;
#define GL_NO_ERROR 0
#define GL_TRIANGLES 4
#define GL_MODELVIEW 0x1700
#define GL_PROJECTION 0x1701
static inline GLenum glGetError(void) { return GL_NO_ERROR; }
static inline void glBegin(GLenum) {}
static inline void glEnd(void) {}
static inline void glVertex3f(float, float, float) {}
static inline void glNormal3f(float, float, float) {}
static inline void glColor3f(float, float, float) {}
static inline void glMatrixMode(GLenum) {}
static inline void glLoadMatrixf(const GLfloat*) {}
static inline void glLoadIdentity(void) {}
#endif
