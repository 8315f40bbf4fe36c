/* Header shim: see GL/gl.h. */
#include "GL/gl.h"
