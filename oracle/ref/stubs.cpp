/*
 * Test infrastructure (oracle build only): link stubs for the two reference
 * pieces that need libraries absent from this machine.
 *
 *  - SubdivisionSurface (reference object/subdivision_surface.cpp) needs
 *    OpenSubdiv.  The synthetic scenes never contain subdivision surfaces,
 *    so finalize() and intersect_rays() are empty.
 *  - Renderer::render (reference renderer/renderer.cpp) writes PNGs through
 *    OpenImageIO.  The oracle driver builds the Film and the
 *    PathTraceIntegrator itself instead.
 */
#include "subdivision_surface.hpp"
#include "renderer.hpp"

void SubdivisionSurface::finalize() {}

void SubdivisionSurface::intersect_rays(Ray*, Ray*, Intersection*, const Range<const Transform*>,
                                        Stack*, const SurfaceShader*, const InstanceID&) const {}

bool Renderer::render(int) {
	return false;
}
