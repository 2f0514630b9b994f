/* Test infrastructure (oracle build only): empty stand-in.  OpenImageIO is
 * only used by the reference's PNG writer (renderer/renderer.cpp), which the
 * oracle build does not compile. */
