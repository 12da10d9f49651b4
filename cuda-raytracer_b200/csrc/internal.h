// Host-side helpers shared between api.cpp and other translation units of the
// library (not part of the C ABI).
#pragma once
#include <string>

#include "../../include/cr.h"
#include "render.h"

namespace cr
{
// Validates a render request against a committed scene and fills the device
// scene view and the render configuration.  Pure host work: no device
// allocation, no synchronisation.  Returns CR_OK or an error code with the
// message in `err`.
int prepare_render( cr_scene *s, const cr_render_desc *desc, DevScene &sc, RenderConfig &cfg, std::string &err );
// The max_bounce a render request resolves to: desc->max_bounce, or the
// scene's (from its kernel's "maxBounce") when the request leaves it at
// UINT32_MAX.  Host work only.
uint32_t effective_max_bounce( const cr_scene *s, const cr_render_desc *desc );
// Records the message returned by cr_last_error() on this thread.
void set_last_error( const std::string &msg );
}  // namespace cr
