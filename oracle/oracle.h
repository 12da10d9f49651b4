/* FP64 CPU oracle for the Radiance path of xlnx/cuda-raytracer.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this library, and only as the checker.
 * The product (the CUDA path behind include/cr.h) never links or calls it.
 *
 * It restates, in double precision, the reference's per-sample Radiance
 * integrator and everything it calls (citations at each function in
 * oracle.cpp), in two estimator modes:
 *   ORC_KOISHI: the reference's semantics exactly, including its quirks
 *               (NEE plus emission on every hit, Lambert weight carrying an
 *               extra cosine, the Glossy/Beckmann lobe as written, the
 *               1024-point mesh light tables, uniform-theta sphere sampling,
 *               the n x (0,1,0) shading frame and 4e-3 offsets);
 *   ORC_MIS:    the corrected estimator the CUDA path also implements
 *               (power-heuristic MIS of BSDF sampling and area-light NEE,
 *               energy-consistent Lambert and Beckmann microfacet BSDFs,
 *               rough dielectrics after Walter et al. 2007, a delta
 *               pass-through for Transparent, Mixed of two leaves, point
 *               lights with 1/r^2 falloff, area-proportional light
 *               sampling, two-sided shading).  orc_render's estimators 2
 *               and 3 run it with BSDF sampling alone and with the light
 *               samples' weights alone, for consistency checks.
 */
#ifndef CR_ORACLE_H
#define CR_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_KOISHI = 0, ORC_MIS = 1 };
/* The reference's debug kernels (src/core/kernel/{normal,visibility,halfVector}.hpp),
 * as orc_render estimators: shading normal * 0.5 + 0.5; 1 where the light-0
 * sample is unoccluded with nonzero radiance; the half-vector angle of the
 * light-0 sample and the view direction, * 2 / pi. */
enum { ORC_AOV_NORMAL = 4, ORC_AOV_VISIBILITY = 5, ORC_AOV_HALFVECTOR = 6 };
enum { ORC_LAMBERT = 0, ORC_GLOSSY = 1, ORC_EMISSION = 2, ORC_TRANSPARENT = 3, ORC_BLACKHOLE = 4,
       ORC_REFRACTION = 5, ORC_GLASS = 6, ORC_MIXED = 7 };
enum { ORC_DIST_BECKMANN = 0, ORC_DIST_COSINE = 1 };
enum { ORC_FAC_CONSTANT = 0, ORC_FAC_FRESNEL = 1 };

typedef struct orc_scene orc_scene;

orc_scene *orc_scene_new(void);
void orc_scene_free(orc_scene *s);

/* params: LAMBERT {R[3], color[3]}; GLOSSY {color[3], roughness, dist};
 * EMISSION {color[3], strength}; TRANSPARENT {color[3]}; BLACKHOLE {};
 * REFRACTION and GLASS {color[3], ior, roughness, dist}; MIXED {fac kind,
 * fac value (Constant) or ior (Fresnel), shader a, shader b} with a and b
 * ids returned earlier.  Returns the shader id (-1 for a bad type or child). */
int orc_add_shader(orc_scene *s, int type, const double *params);
/* A pointLight asset (position, color, strength); point lights precede the
 * area lights in the light list.  Returns its index among point lights. */
int orc_add_point_light(orc_scene *s, const float *pos, const double *color, double strength);
/* Shader::execute of shader id with k scripted draws u (target 0
 * compute_f_by_wi_wo, 1 sample_wi_f_by_wo; wi is in/out).  Writes f[3] and
 * the emission the executed shader sets; returns the number of draws made
 * (draws past k read 0.5). */
int orc_shade(const orc_scene *s, int shader, int target, const double *wo, double *wi, const double *u, int k,
              double *f, double *emission);
/* ORC_MIS BSDF of shader id (a leaf or a Mixed of two leaves) in the local
 * frame, wo.z > 0; entering: wo lies outside the surface as built.  eval: f
 * and pdf of wi; sample (u = {u1, u2, selection}): wi, weight f|cos|/pdf and
 * pdf; returns 1 for the delta (Transparent) direction, whose weight is its
 * colour and which has no density. */
void orc_mis_eval(const orc_scene *s, int shader, const double *wo, const double *wi, int entering, double *f,
                  double *pdf);
int orc_mis_sample(const orc_scene *s, int shader, const double *wo, int entering, const double *u, double *wi,
                   double *weight, double *pdf);
/* Primitives are numbered in the order they are added. Returns the prim id. */
int orc_add_mesh(orc_scene *s, const float *v, uint32_t nv, const float *n, const uint32_t *idx,
                 uint32_t nt, int shader);
int orc_add_sphere(orc_scene *s, const float *center, float radius, int shader);
void orc_set_camera(orc_scene *s, const float *pos, const float *target, const float *up, float fovx);
/* CameraConfig::lens: 0 pinhole, 1 orthographic (lens.hpp:40-66). */
void orc_set_lens(orc_scene *s, int lens);
/* Builds the BVH and the light list; light_seed is the 48-bit state the
 * 1024-point tables are drawn from (ORC_KOISHI). */
int orc_finalize(orc_scene *s, uint64_t light_seed);

int orc_num_lights(const orc_scene *s);
/* 1024 x {p.xyz, n.xyz} (float) of light l if it is a mesh light; returns the
 * table's area pdf, or -1 for a sphere light. */
double orc_light_table(const orc_scene *s, int l, float *pts);

/* rays: n x {o.xyz, d.xyz, tmax} (float, d as given).  Closest hit in FP64
 * with the reference's triangle and sphere tests; prim -1 on a miss. */
void orc_trace(const orc_scene *s, const float *rays, uint64_t n, int32_t *prim, int32_t *tri,
               double *t, double *u, double *v);
/* FP64 intersection of one ray with one given triangle (no bounds on u, v). */
void orc_ray_triangle(const orc_scene *s, const float *ray, int prim, int tri, double *t, double *u,
                      double *v);
/* segs: n x {o.xyz, d.xyz, t}: the reference's Scene::intersect(Seg). */
void orc_occluded(const orc_scene *s, const float *segs, uint64_t n, uint8_t *out);

/* Per-pixel film over the window [x0,x1) x [y0,y1) of a W x H image:
 * sum, sum of squares (3 doubles each) and the number of finite samples.
 * Returns -1 for a bad window, -2 when ORC_MIS meets a point light or a
 * shader other than Lambert, Beckmann Glossy and Emission. */
int orc_render(const orc_scene *s, uint32_t W, uint32_t H, uint32_t spp, uint32_t max_bounce,
               int estimator, uint64_t seed, uint32_t threads, uint32_t x0, uint32_t y0,
               uint32_t x1, uint32_t y1, double *sum, double *sumsq, uint32_t *count);

/* BSDF in the local shading frame (z = normal).  shader params as in
 * orc_add_shader.  eval: f (rgb) and pdf of wi; sample: wi, weight
 * (f*|cos|/pdf), pdf from uniforms u[3]. */
void orc_bsdf_eval(int estimator, int type, const double *params, const double *wo,
                   const double *wi, double *f, double *pdf);
void orc_bsdf_sample(int estimator, int type, const double *params, const double *wo,
                     const double *u, double *wi, double *weight, double *pdf);

/* Known-answer helpers for the reference's own unit tests. */
int orc_seg_box(const float *seg7, const float *bmin, const float *bmax);
int orc_sphere_hit(const float *center, float radius, const float *ray6, double *t);

#ifdef __cplusplus
}
#endif
#endif
