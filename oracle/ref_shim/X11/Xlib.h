/* Type-only stand-in for <X11/Xlib.h>, used solely by the oracle's build of the
 * reference CPU fitter.  The reference's texture header reaches the OpenGL loader
 * header, which names a handful of X11/GLX types in declarations.  Nothing on the
 * fitting path calls or links X11 or OpenGL, so opaque declarations suffice. */
#ifndef SVF_ORACLE_XLIB_SHIM_H
#define SVF_ORACLE_XLIB_SHIM_H
typedef struct _XDisplay Display;
typedef unsigned long XID;
typedef XID Window;
typedef XID Pixmap;
typedef XID Colormap;
typedef XID Font;
typedef XID Cursor;
typedef int Bool;
typedef int Status;
typedef struct { void* visual; unsigned long visualid; int screen; int depth; int c_class;
                 unsigned long red_mask, green_mask, blue_mask; int colormap_size; int bits_per_rgb; } XVisualInfo;
typedef struct __GLXcontextRec* GLXContext;
typedef struct __GLXFBConfigRec* GLXFBConfig;
typedef XID GLXDrawable;
typedef XID GLXPbuffer;
typedef XID GLXPixmap;
typedef XID GLXWindow;
#endif
