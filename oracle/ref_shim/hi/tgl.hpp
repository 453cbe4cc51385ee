// The reference's OpenGL preview (the Render() methods) is left out of the
// oracle: these empty functions let those methods compile and do nothing.
// Nothing here draws anything or loads a graphics library.
#pragma once
#include <hi/lang.hpp>
#define GL_TRIANGLES 0
#define GL_LIGHTING 0
#define GL_BLEND 0
#define GL_FRONT_AND_BACK 0
#define GL_AMBIENT_AND_DIFFUSE 0
#define GL_SPECULAR 0
#define GL_SRC_ALPHA 0
#define GL_ONE_MINUS_SRC_ALPHA 0
#define GL_SHININESS 0
#define GL_PROJECTION 0
#define GL_MODELVIEW 0
#define GL_COMPILE 0
typedef float GLfloat;
#define XYZREF_NOGL(name) \
  template <class... A>   \
  inline void name(A const &...) {}
XYZREF_NOGL(glBegin)
XYZREF_NOGL(glEnd)
XYZREF_NOGL(glEnable)
XYZREF_NOGL(glDisable)
XYZREF_NOGL(glCallList)
XYZREF_NOGL(glMatrixMode)
XYZREF_NOGL(glLoadIdentity)
XYZREF_NOGL(gluPerspective)
XYZREF_NOGL(gluLookAt)
XYZREF_NOGL(glPushMatrix)
XYZREF_NOGL(glPopMatrix)
XYZREF_NOGL(glutSolidSphere)
XYZREF_NOGL(glNewList)
XYZREF_NOGL(glEndList)
XYZREF_NOGL(glBlendFunc)
inline unsigned int glGenLists(int) { return 0u; }
namespace hi {
XYZREF_NOGL(glNormal)
XYZREF_NOGL(glMaterial)
XYZREF_NOGL(glTranslate)
XYZREF_NOGL(glVertex)
template <int N, class... A>
inline void glVertex(A const &...) {}
}  // namespace hi
#undef XYZREF_NOGL
