// No-op OpenGL surface for compiling the reference headlessly.
// TEST INFRASTRUCTURE (reference cross-check build only).
#pragma once
typedef unsigned int GLuint;
typedef int GLint;
typedef int GLsizei;
typedef unsigned int GLenum;
typedef float GLfloat;
typedef unsigned char GLboolean;
typedef long GLsizeiptr;
#define GL_ARRAY_BUFFER 0x8892
#define GL_ELEMENT_ARRAY_BUFFER 0x8893
#define GL_FLOAT 0x1406
#define GL_FALSE 0
#define GL_TRUE 1
#define GL_DYNAMIC_DRAW 0x88E8
#define GL_POINTS 0x0000
#define GL_LINES 0x0001
#define GL_UNSIGNED_INT 0x1405
#define GL_VERTEX_SHADER 0x8B31
#define GL_FRAGMENT_SHADER 0x8B30
inline GLint glGetUniformLocation(GLuint, const char*) { return -1; }
inline void glGenVertexArrays(GLsizei n, GLuint* a) { for (GLsizei i = 0; i < n; ++i) a[i] = 0; }
inline void glGenBuffers(GLsizei n, GLuint* a) { for (GLsizei i = 0; i < n; ++i) a[i] = 0; }
inline void glBindVertexArray(GLuint) {}
inline void glBindBuffer(GLenum, GLuint) {}
inline void glEnableVertexAttribArray(GLuint) {}
inline void glVertexAttribPointer(GLuint, GLint, GLenum, GLboolean, GLsizei, const void*) {}
inline void glDeleteBuffers(GLsizei, const GLuint*) {}
inline void glDeleteVertexArrays(GLsizei, const GLuint*) {}
inline void glDeleteProgram(GLuint) {}
inline void glUseProgram(GLuint) {}
inline void glPointSize(GLfloat) {}
inline void glLineWidth(GLfloat) {}
inline void glBufferData(GLenum, GLsizeiptr, const void*, GLenum) {}
inline void glUniform3fv(GLint, GLsizei, const GLfloat*) {}
inline void glUniform1f(GLint, GLfloat) {}
inline void glUniform4f(GLint, GLfloat, GLfloat, GLfloat, GLfloat) {}
inline void glDrawArrays(GLenum, GLint, GLsizei) {}
inline void glDrawElements(GLenum, GLsizei, GLenum, const void*) {}
