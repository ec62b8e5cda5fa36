// No-op OpenGL stand-in (written for this project) so the reference's
// src/renderer/octree.cpp compiles without a graphics stack.  Test
// infrastructure only: every call is a no-op except glGetIntegerv, which
// reports a texture-buffer limit large enough that Octree never clamps.
#pragma once
#include <cstddef>
#include <cstdint>

typedef unsigned int GLuint;
typedef int GLint;
typedef int GLsizei;
typedef unsigned int GLenum;
typedef float GLfloat;
typedef unsigned char GLboolean;
typedef ptrdiff_t GLintptr;
typedef ptrdiff_t GLsizeiptr;

#define GL_TEXTURE_BUFFER 0x8C2A
#define GL_DYNAMIC_DRAW 0x88E8
#define GL_R32UI 0x8236
#define GL_TEXTURE0 0x84C0
#define GL_MAX_TEXTURE_BUFFER_SIZE 0x8C2B

inline void glGetIntegerv(GLenum, GLint* v) { *v = 1 << 30; }
inline void glGenBuffers(GLsizei n, GLuint* b) { for (GLsizei i = 0; i < n; i++) b[i] = 1u + i; }
inline void glGenTextures(GLsizei n, GLuint* t) { for (GLsizei i = 0; i < n; i++) t[i] = 1u + i; }
inline void glBindBuffer(GLenum, GLuint) {}
inline void glBufferData(GLenum, GLsizeiptr, const void*, GLenum) {}
inline void glBufferSubData(GLenum, GLintptr, GLsizeiptr, const void*) {}
inline void glBindTexture(GLenum, GLuint) {}
inline void glTexBuffer(GLenum, GLenum, GLuint) {}
inline void glDeleteBuffers(GLsizei, const GLuint*) {}
inline void glDeleteTextures(GLsizei, const GLuint*) {}
inline void glActiveTexture(GLenum) {}
inline GLint glGetUniformLocation(GLuint, const char*) { return 0; }
inline void glUniform1i(GLint, GLint) {}
inline void glUniform1ui(GLint, GLuint) {}
