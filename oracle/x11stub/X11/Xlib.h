/* Compile-only stand-in for <X11/Xlib.h>, used only to compile the reference's
 * CPU demag sources for the oracle (the reference header BorisLib/Funcs_Files_Linux.h
 * includes Xlib for a clipboard helper that the oracle never calls).
 * Declarations only: nothing here is ever executed or linked. */
#pragma once
typedef struct _XDisplay Display;
typedef unsigned long Window;
typedef unsigned long Atom;
typedef unsigned long Time;
typedef int Bool;
typedef struct { int type; struct { Atom selection; Atom property; } xselection; struct { Atom atom; int state; } xproperty; char pad[192]; } XEvent;
#define True 1
#define False 0
#define None 0L
#define CurrentTime 0L
#define PropertyChangeMask (1L << 22)
#define SelectionNotify 31
#define PropertyNotify 28
#define PropertyNewValue 0
#define AnyPropertyType 0L
#ifdef __cplusplus
extern "C" {
#endif
Atom XInternAtom(Display *, const char *, Bool);
int XSelectInput(Display *, Window, long);
int XConvertSelection(Display *, Atom, Atom, Atom, Window, Time);
int XNextEvent(Display *, XEvent *);
int XGetWindowProperty(Display *, Window, Atom, long, long, Bool, Atom, Atom *, int *, unsigned long *, unsigned long *, unsigned char **);
int XFree(void *);
int XDeleteProperty(Display *, Window, Atom);
Display *XOpenDisplay(const char *);
Window XCreateSimpleWindow(Display *, Window, int, int, unsigned int, unsigned int, unsigned int, unsigned long, unsigned long);
Window XDefaultRootWindow(Display *);
#define DefaultRootWindow(d) XDefaultRootWindow(d)
unsigned long XBlackPixel(Display *, int);
#define BlackPixel(d, s) XBlackPixel(d, s)
int XDefaultScreen(Display *);
#define DefaultScreen(d) XDefaultScreen(d)
int XDestroyWindow(Display *, Window);
int XCloseDisplay(Display *);
#ifdef __cplusplus
}
#endif
