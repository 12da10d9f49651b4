// Compile check of the Tracer plugin that the integration guide shows a
// maintainer adding to the reference (test infrastructure, syntax and types
// only; the plugin's text comes from the guide's C++ blocks).  The
// two accessors of Sphere's private centre and radius are declared here, as
// the plugin's text leaves them to the maintainer.
#include <map>
#include <string>
#include <vector>

#include <core/light/pointLight.hpp>
#include <core/primitive/sphere.hpp>
#include <core/tracer/tracer.hpp>

namespace koishi
{
namespace core
{
#include "tocfg.hpp"
const float *sphere_center( const Sphere &s );
float sphere_radius( const Sphere &s );
}  // namespace core
}  // namespace koishi

#include "plugin.hpp"
