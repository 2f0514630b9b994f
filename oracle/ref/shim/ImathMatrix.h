/* Test infrastructure (oracle build only): empty stand-in.  The reference
 * selects its own Matrix44 (reference math/matrix.hpp:17 `#if 1`), so no
 * IlmBase matrix is needed. */
