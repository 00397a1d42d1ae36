// sg_integrator.cuh — the integrator's per-path state and one iteration of
// trace()'s loop (pathtrace.wgsl:1347-1617), split into extend() (the
// closest hit) and the two vertex kinds it leads to, ring_vertex() and
// surface_vertex(). The per-pixel megakernel runs them back to back through
// step(); the wavefront integrator runs each as its own stage over queues of
// paths. Both therefore execute the same arithmetic on every path.
#pragma once

#include "sg_adjoint.cuh"
#include "sg_air.cuh"
#include "sg_device.cuh"
#include "sg_internal.h"
#include "sg_landscape.cuh"

namespace sg {

namespace {

constexpr int kTile = 16;
constexpr int kThreads = 256;

// The state trace() (pathtrace.wgsl:1347-1617) carries from one path vertex
// to the next.
struct Path {
    Ray ray;
    Ray previous_vertex;  // the last scattering vertex (null crossings keep it)
    float3 throughput;
    float3 radiance;
    float3 ring_base;
    float previous_pdf;
    float ring_cap;
    uint32_t depth;
    uint32_t null_crossings;
    uint32_t shine_body;
    uint32_t iterations;
    uint32_t rng;
    bool point_gained;
    float3 backdrop;  // Milky Way radiance reached by an unscattered camera path
    // Host air (pathtrace.wgsl:1361-1368): the previous vertex lies in the
    // air; the previous vertex was a sky-lit local surface.
    bool in_air;
    bool sky_on_escape;
    uint32_t sample;  // the sample's index in its dispatch (its counts.y offset)
    // Checkpoints the forward stored for this sample (sg_set_checkpoints):
    // bit 0 some were stored, bit 1 one did not fit (the sample then replays
    // from its seed).
    uint32_t ckpt;
};

// camera_direction (pathtrace.wgsl:1619-1626).
template <bool C, bool L, bool F>
__device__ __forceinline__ float3 camera_direction(const sg_settings *s, Counter<C, L, F> K, uint32_t x, uint32_t y,
                                                   uint32_t &rng) {
    const float jx = rnd(K, rng);
    const float jy = rnd(K, rng);
    const float u = ((float)x + jx) / s->g.viewport[0];
    const float v = ((float)y + jy) / s->g.viewport[1];
    const float tangent = s->g.cam_forward[3];
    return normalize(f3((2.0f * u - 1.0f) * tangent * s->g.viewport[3], (1.0f - 2.0f * v) * tangent, -1.0f));
}

// Sample `smp` of a pixel: seeding (pathtrace.wgsl:1656), the jittered
// camera ray, and trace()'s initial state.
template <bool C, bool L, bool F>
__device__ __forceinline__ void start_path(Path &p, const sg_settings *s, Counter<C, L, F> K, uint32_t pixel, uint32_t x,
                                           uint32_t y, uint32_t smp) {
    p.rng = hash_u32(pixel ^ hash_u32(s->sampling[0] + smp + 0x9e3779b9u));
    const float3 d = camera_direction(s, K, x, y, p.rng);
    p.ray = Ray{f3(0.0f, 0.0f, 0.0f), d, kMiss};
    p.previous_vertex = p.ray;
    p.throughput = f3(1.0f, 1.0f, 1.0f);
    p.radiance = f3(0.0f, 0.0f, 0.0f);
    p.ring_base = f3(0.0f, 0.0f, 0.0f);
    p.previous_pdf = 0.0f;
    p.ring_cap = 1.0e30f;
    p.depth = 0;
    p.null_crossings = 0;
    p.shine_body = kMiss;
    p.iterations = 0;
    p.point_gained = false;
    p.backdrop = f3(0.0f, 0.0f, 0.0f);
    p.in_air = false;
    p.sky_on_escape = false;
    p.sample = smp;
    p.ckpt = 0;
}

// The ring-indirect cap after the loop (pathtrace.wgsl:1609-1615); W holds
// the backdrop's luminance (for exposure metering and the display).
__device__ __forceinline__ float4 finish_path(const Path &p) {
    float3 radiance = p.radiance;
    if (p.ring_cap < 1.0e29f) {
        const float3 indirect = radiance - p.ring_base;
        const float l = luminance(indirect);
        if (l > p.ring_cap) radiance = p.ring_base + indirect * (p.ring_cap / l);
    }
    return make_float4(radiance.x, radiance.y, radiance.z, luminance(p.backdrop));
}

// A camera path that escapes unscattered (pathtrace.wgsl:1494-1508): the
// catalogue discs of its direction and the Milky Way, through its
// throughput (null ring crossings attenuate both). Scattered paths see
// neither. Draws no random numbers.
struct SkyTerms {
    float3 env;       // throughput x catalogue discs
    float3 backdrop;  // Milky Way x throughput
};
// Out of line: it runs only where a camera path escapes, and keeps the
// extend stage's register allocation that of the sky-less frames.
static __device__ __noinline__ SkyTerms sky_terms(const TraceParams *P, float3 dir, float3 throughput) {
    return SkyTerms{throughput * environment(P, dir), milky_way(P, dir) * throughput};
}
__device__ __forceinline__ void sky_miss(const Scene &S, Path &p) {
    if (!S.p->sky_on || p.depth != 0u) return;
    const SkyTerms t = sky_terms(S.p, p.ray.d, p.throughput);
    p.radiance = p.radiance + t.env;
    p.backdrop = t.backdrop;
    p.radiance = p.radiance + p.backdrop;
}

// The backdrop accumulation (pathtrace.wgsl:1654-1674): the dispatch's mean
// folded into the running mean.
__device__ __forceinline__ void fold_backdrop(const TraceParams &P, uint32_t pixel, float3 sum) {
    const float z = (float)P.s.counts[2];
    float3 mean = sum / z;
    if (P.s.counts[1] > 0u) {
        const float4 old = P.backdrop[pixel];
        const float w = z / (float)(P.s.counts[1] + P.s.counts[2]);
        mean = f3(old.x + (mean.x - old.x) * w, old.y + (mean.y - old.y) * w, old.z + (mean.z - old.z) * w);
    }
    P.backdrop[pixel] = make_float4(mean.x, mean.y, mean.z, 0.0f);
}

// The host air at the start of an iteration (pathtrace.wgsl:1387-1414):
// extinction of a continuation that left the air for a celestial surface
// or a ring, and on the camera ray its in-scatter and view transmittance.
template <bool C, bool L, bool F>
__device__ __forceinline__ void air_extend(const Scene &S, Counter<C, L, F> K, Path &p, const Hit &hit,
                                           const RingHit &ring) {
    if (p.in_air) {
        p.in_air = false;
        const uint32_t host = (uint32_t)S.s->g.atmo_params[3] - 1u;
        if (ring.index != kMiss || (hit.index < kLocalBase && hit.index != host))
            p.throughput = p.throughput * air_transmittance(S, p.ray, p.ray.d);
    }
    if (p.iterations == 1u) {
        float limit = 1.0e30f;
        if (hit.index != kMiss) limit = hit.t;
        if (ring.index != kMiss) limit = fminf(limit, ring.t);
        const AirScatter a = atmosphere(S, K, p.ray.o, p.ray.d, limit, p.rng, S.s->counts[1] + p.sample);
        p.radiance = p.radiance + p.throughput * a.inscatter;
        p.throughput = p.throughput * a.transmittance;
        p.rng = a.rng;
    }
}

// What extend() finds along a path's current ray.
struct Extension {
    Hit hit;          // closest body or landscape hit (after the disc test)
    RingHit ring;     // closest ring crossing before it, or a miss
    float disc_scale; // point-disc scale of a depth-0 camera ray
};

// First part of one iteration of trace()'s loop (pathtrace.wgsl:1380-1414):
// the iteration bound, the closest hit, the depth-0 point-disc test and the
// closest ring crossing before the hit. Returns false when the path has
// ended at the bound.
// `cull`: the tile's masks for a camera ray (its first extend), else
// kTestAll.
template <bool C, bool L, bool F, class G>
__device__ __forceinline__ bool extend(const Scene &S, Counter<C, L, F> K, Path &p, G &grad, Extension &e,
                                       Cull cull = kTestAll) {
    const sg_settings *s = S.s;
    const uint32_t max_vertices = s->counts[3];
    const uint32_t n_bodies = s->counts[0];
    // Static bound: each of at most max_vertices vertices is preceded by at
    // most n_bodies + 1 null crossings, so valid inputs never reach it.
    if (++p.iterations > max_vertices * (n_bodies + 2u) + 1u) return false;
    if constexpr (G::adjoint) grad.iteration = p.iterations;
    K.add(&Events::vertices);
    e.hit = closest_hit(S, K, p.ray, cull);
    e.disc_scale = 1.0f;
    if (p.depth == 0u && p.null_crossings == 0u && s->background[3] > 0.0f) {
        const DiscHit disc = point_disc_hit(S, K, p.ray, e.hit, p.rng, cull);
        e.hit = disc.hit;
        e.disc_scale = disc.scale;
        p.rng = disc.rng;
    }
    e.ring = closest_ring(S, K, p.ray, e.hit.t, cull);
    if constexpr (G::air) {
        if (S.p->air_on) air_extend(S, K, p, e.hit, e.ring);
    }
    return true;
}

// A ring event (pathtrace.wgsl:1415-1493) at `ring`: next-event estimation
// of every star through the slab, then the null-or-scatter decision.
// Returns true when the path has ended.
template <bool C, bool L, bool F, class G>
__device__ __forceinline__ bool ring_vertex(const Scene &S, Counter<C, L, F> K, Path &p, const RingHit &ring,
                                            G &grad) {
    const sg_settings *s = S.s;
    const uint32_t max_vertices = s->counts[3];
    const uint32_t n_bodies = s->counts[0];
    const float gain = s->background[3];
    const uint32_t n_lights = light_count(s);
    Ray &ray = p.ray;
    uint32_t &rng = p.rng;
    float3 &throughput = p.throughput;
    float3 &radiance = p.radiance;
    uint32_t &depth = p.depth;
    uint32_t &null_crossings = p.null_crossings;
    bool &point_gained = p.point_gained;
    uint32_t &shine_body = p.shine_body;
    float &previous_pdf = p.previous_pdf;
    Ray &previous_vertex = p.previous_vertex;
    float &ring_cap = p.ring_cap;
    float3 &ring_base = p.ring_base;
    {
        {
            K.add(&Events::ring_events);
            const uint32_t ri = ring.index;
            if (depth == 0u && !point_gained && gain > 0.0f) {
                point_gained = true;
                throughput = throughput * point_gain(s, b_radius(S, ri) * bf(S, ri, kRingParams).x, ring.t);
            }
            const float3 n = xyz(bf(S, ri, kRingPlane));
            const Optics optics = ring_optics(S, ri, ring.p);
            const float mu_out = dot(-ray.d, n);
            const float transmission = ring_transmission_tau(ray.d, n, optics.tau);
            const float scatter_probability = one_minus_exp(optics.tau / fmaxf(fabsf(mu_out), 1.0e-7f));
            const float bsdf_pdf = scatter_probability / (4.0f * kPi);
            const bool last_vertex = depth + 1u == max_vertices;
            float ring_mis = 1.0f;
            if (shine_body == ri && null_crossings == 0u) {
                const float cos_ring = fmaxf(fabsf(dot(ray.d, n)), 1.0e-6f);
                const float shine_pdf = ring.t * ring.t / (ring_area(S, ri) * cos_ring);
                ring_mis = power_weight(previous_pdf, shine_pdf);
            }
            shine_body = kMiss;
            [[maybe_unused]] RingVertexGrad vg{kNoParam, 0.0f, 0.0f};
            if constexpr (G::adjoint) {
                vg = ring_vertex_grad(S, ri, ring.p, optics.tau, mu_out);
                if (!grad.pass2) {
                    grad.lit_sum = f3(0.0f, 0.0f, 0.0f);
                    grad.lit_vis_sum = f3(0.0f, 0.0f, 0.0f);
                }
            }
            float unshadowed = 0.0f, direct = 0.0f;
            #pragma unroll 1
            for (uint32_t slot = 0; slot < n_lights; ++slot) {
                const uint32_t i = light_index(s, slot);
                const float4 material = bf(S, i, kMaterial);
                if (material.w < 0.5f || optics.tau == 0.0f) continue;
                const LightSample light = sample_light(S, K, Ray{ring.p, n, ri}, i, rng);
                rng = light.rng;
                const float mu_in = dot(light.d, n);
                float visibility;
                [[maybe_unused]] Visibility vis;
                if constexpr (G::adjoint) {
                    vis = light_visibility_grad(S, K, ring_origin(S, ri, ring.p, light.d), i, true);
                    visibility = vis.v;
                } else {
                    visibility = light_visibility(S, K, ring_origin(S, ri, ring.p, light.d), i);
                }
                const float weight = last_vertex ? 1.0f : power_weight(light.pdf, bsdf_pdf);
                const float3 lit = throughput * ring_bsdf(optics, mu_out, mu_in) * xyz(material) *
                                   (fabsf(mu_in) / light.pdf);
                radiance = radiance + lit * (visibility * weight * ring_mis);
                if constexpr (G::adjoint) {
                    ring_light_grad(S, grad, ri, optics, mu_out, mu_in, i, lit, vis, weight, ring_mis, last_vertex, vg);
                    if (!grad.pass2) {
                        grad.lit_sum = grad.lit_sum + lit;
                        grad.lit_vis_sum = grad.lit_vis_sum + lit * visibility;
                    }
                }
                const float l = luminance(lit);
                unshadowed += l;
                direct += l * visibility;
            }
            if (rnd(K, rng) < transmission) {
                // Null event: no depth consumed, MIS stays with the last vertex.
                if constexpr (G::adjoint) {
                    ring_null_grad(S, grad, ri, ring.p, ray.d);
                }
                ray = ring_origin(S, ri, ring.p, ray.d);
                null_crossings += 1u;
                return null_crossings > n_bodies;
            }
            if (last_vertex || scatter_probability == 0.0f) return true;
            if (ring_cap > 1.0e29f) {
                ring_cap = fmaxf(direct, kRingIndirectCap * unshadowed);
                ring_base = radiance;
                if constexpr (G::adjoint) {
                    if (!grad.pass2)
                        record_capture(grad, p.iterations, ring_cap, direct >= kRingIndirectCap * unshadowed, radiance);
                }
            }
            const float z = 1.0f - 2.0f * rnd(K, rng);
            float sp, cp;
            sincos_turn(rnd(K, rng), &sp, &cp);
            const float radial = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            const float3 direction = basis_direction(n, radial * cp, radial * sp, z);
            throughput = throughput * ring_bsdf(optics, mu_out, z) * (fabsf(z) / bsdf_pdf);
            if constexpr (G::adjoint) {
                ring_scatter_grad(S, grad, ri, optics, mu_out, z, vg, transmission, ray.d);
            }
            previous_pdf = bsdf_pdf;
            if constexpr (G::air) p.sky_on_escape = false;
            ray = ring_origin(S, ri, ring.p, direction);
            previous_vertex = ray;
            depth += 1u;
            null_crossings = 0u;
            if (depth >= 3u) {
                const float survival = clampf(max3(throughput), 0.05f, 0.95f);
                const bool survived = !(rnd(K, rng) >= survival);
                if constexpr (G::adjoint) {
                    if (!grad.pass2) record_roulette(grad, p.iterations, throughput, survival, survived, radiance);
                }
                if (!survived) return true;
                throughput = throughput / survival;
            }
            return false;
        }
    }
}

// The rest of the iteration when no ring crossing comes first
// (pathtrace.wgsl:1494-1607): environment miss, emitter hit with MIS, or a
// surface vertex with next-event estimation, ringshine and the cosine
// bounce. Returns true when the path has ended.
template <bool C, bool L, bool F, class G>
__device__ __forceinline__ bool surface_vertex(const Scene &S, Counter<C, L, F> K, Path &p, const Hit &hit,
                                               float disc_scale, G &grad) {
    const sg_settings *s = S.s;
    const uint32_t max_vertices = s->counts[3];
    const float gain = s->background[3];
    const uint32_t n_lights = light_count(s);
    Ray &ray = p.ray;
    uint32_t &rng = p.rng;
    float3 &throughput = p.throughput;
    float3 &radiance = p.radiance;
    uint32_t &depth = p.depth;
    uint32_t &null_crossings = p.null_crossings;
    bool &point_gained = p.point_gained;
    uint32_t &shine_body = p.shine_body;
    float &previous_pdf = p.previous_pdf;
    Ray &previous_vertex = p.previous_vertex;
    {
        // Miss: the sky backdrop of an unscattered camera path (the adjoint
        // does not differentiate it; sg_backward rejects such frames).
        if (hit.index == kMiss) {
            if constexpr (G::air) {
                if (p.sky_on_escape) radiance = radiance + throughput * surface_sky_lookup(S, ray.d);
            }
            if constexpr (G::sky) sky_miss(S, p);
            return true;
        }

        const uint32_t bi = hit.index;
        // Local ids (host sphere, terrain, props) never index the bodies;
        // the landscape-free instantiation (L == false) never sees them.
        const bool local = L && bi >= kLocalBase;
        throughput = throughput * disc_scale;
        if (!local && bf(S, bi, kMaterial).w > 0.5f) {
            // Emitter hit with MIS against the previous vertex's light sample.
            float weight = 1.0f;
            if (depth > 0u) {
                const float3 oc = relative_center(S, previous_vertex, bi);
                const float light_pdf = 1.0f / (kTau * cone_width_oc(oc, b_radius(S, bi)));
                weight = power_weight(previous_pdf, light_pdf);
            }
            radiance = radiance + throughput * xyz(bf(S, bi, kMaterial)) * weight;
            if constexpr (G::adjoint) {
                emitter_grad(grad, bi, throughput * xyz(bf(S, bi, kMaterial)) * weight, weight, depth > 0u);
            }
            return true;
        }
        K.add(&Events::surface_events);
        float3 normal;
        Ray outgoing;
        if (local) {
            // Metre-scale surface: bumped shading normal and the 5 mm
            // offset origin (ground.wgsl:633-662).
            if constexpr (L) {
                normal = landscape_shading_normal(S, ray, hit.t, bi, hit.n);
                outgoing = landscape_outgoing<F>(S, ray, hit.t, bi, hit.n);
            }
        } else {
            const float radius = b_radius(S, bi);
            if (depth == 0u && !point_gained && gain > 0.0f) {
                point_gained = true;
                const float extent = radius * fmaxf(1.0f, bf(S, bi, kRingParams).x);
                throughput = throughput * point_gain(s, extent, hit.t);
            }
            normal = sphere_normal(S, ray, bi, hit.delta);
            // Celestial surfaces keep a body-relative origin.
            outgoing = Ray{normal * (radius * (1.0f + 2.0e-6f)), normal, bi};
        }
        // The guided ground sampler (src/guided_ground.rs:38-48): a camera
        // ray's local surface under air picks a reflector (main random
        // stream) to propose half of its continuations toward.
        [[maybe_unused]] Reflector ground_reflector{kMiss, 0.0f};
        bool guided = false;
        if constexpr (G::air && L) {
            if (S.p->guided_ground && local && depth == 0u && s->g.atmo_params[3] > 0.5f) {
                ground_reflector = sample_reflector(S, K, camera_origin(S, outgoing), rng);
                guided = ground_reflector.index != kMiss;
            }
        }
        const bool last_vertex = depth + 1u == max_vertices;
        // The adjoint needs the albedo (and its parameter) before the light
        // loop; the forward evaluates it after, as the WGSL does.
        [[maybe_unused]] float3 albedo_g = f3(0.0f, 0.0f, 0.0f);
        [[maybe_unused]] GradEntry albedo_e = no_entry();
        if constexpr (G::adjoint) {
            if constexpr (L) {
                albedo_g = local ? landscape_albedo(S, ray, hit.t, bi, hit.n) : surface_albedo<G::air>(S, bi, normal);
            } else {
                albedo_g = surface_albedo<G::air>(S, bi, normal);
            }
            albedo_e = albedo_entry<L>(S, grad.inv, ray, hit.t, bi, albedo_g);
        }
        float3 direct_light = f3(0.0f, 0.0f, 0.0f);
        #pragma unroll 1
            for (uint32_t slot = 0; slot < n_lights; ++slot) {
            const uint32_t i = light_index(s, slot);
            const float4 light_material = bf(S, i, kMaterial);
            if (light_material.w < 0.5f) continue;
            const LightSample sample = sample_light(S, K, outgoing, i, rng);
            rng = sample.rng;
            const float cosine = fmaxf(dot(normal, sample.d), 0.0f);
            if (cosine <= 0.0f) continue;
            outgoing.d = sample.d;
            float visibility;
            [[maybe_unused]] Visibility vis;
            if constexpr (G::adjoint) {
                vis = light_visibility_grad(S, K, outgoing, i, true);
                visibility = vis.v;
            } else {
                visibility = light_visibility(S, K, outgoing, i);
            }
            if (visibility > 0.0f) {
                const float bsdf_pdf = cosine / kPi;
                // MIS against the full continuation density (the guided
                // mixture's where it applies; src/guided_ground.rs:50-57).
                float path_pdf = bsdf_pdf;
                if constexpr (G::air && L) {
                    if (guided) path_pdf = 0.5f * (bsdf_pdf + ground_reflector_pdf(S, K, outgoing));
                }
                const float weight = last_vertex ? 1.0f : power_weight(sample.pdf, path_pdf);
                float3 color = xyz(light_material);
                if constexpr (G::air) {
                    if (S.p->air_on) color = color * air_transmittance(S, outgoing, sample.d);
                }
                direct_light = direct_light + color * (bsdf_pdf * weight * visibility / sample.pdf);
                if constexpr (G::adjoint)
                    surface_light_grad(grad, albedo_e, i,
                                       throughput * albedo_g * xyz(light_material) *
                                           (bsdf_pdf * weight * visibility / sample.pdf),
                                       vis);
            }
        }
        float3 albedo;
        if constexpr (L) {
            albedo = local ? landscape_albedo(S, ray, hit.t, bi, hit.n) : surface_albedo<G::air>(S, bi, normal);
        } else {
            albedo = surface_albedo<G::air>(S, bi, normal);
        }
        radiance = radiance + throughput * albedo * direct_light;
        const bool shines = !local && S.p->ringshine && has_ring(S, bi);
        if (shines) {
            Shine shine;
            if constexpr (G::adjoint)
                shine = ringshine_grad(S, K, bi, outgoing.o, normal, last_vertex, rng, grad, throughput * albedo,
                                       albedo_e);
            else
                shine = ringshine(S, K, bi, outgoing.o, normal, last_vertex, rng);
            rng = shine.rng;
            radiance = radiance + throughput * albedo * shine.radiance;
        }
        // Sky light of local surfaces (pathtrace.wgsl:1578-1584): an explicit
        // sample at the depth limit, else the continuation's escape.
        bool sky_lit = false;
        if constexpr (G::air && L) {
            sky_lit = local && s->g.ground_counts[1] != 0u && s->g.atmo_params[3] > 0.5f;
            if (sky_lit && last_vertex) {
                const SkySample sky = surface_sky(S, K, outgoing, normal, rng);
                rng = sky.rng;
                radiance = radiance + throughput * albedo * sky.radiance;
            }
        }
        shine_body = (local || !S.p->ringshine) ? kMiss : bi;
        if (last_vertex) return true;
        const float u = rnd(K, rng);
        float sp, cp;
        sincos_turn(rnd(K, rng), &sp, &cp);
        const float cosine = sqrtf(1.0f - u);
        const float su = sqrtf(u);
        outgoing.d = basis_direction(normal, su * cp, su * sp, cosine);
        previous_pdf = cosine / kPi;
        float path_weight = 1.0f;
        if constexpr (G::air && L) {
            // src/guided_ground.rs:59-76: half the continuations toward the
            // reflector, weighted by cosine density over the mixture's.
            if (guided) {
                if (rnd(K, rng) < 0.5f) {
                    const LightSample toward = sample_light(S, K, outgoing, ground_reflector.index, rng);
                    rng = toward.rng;
                    outgoing.d = toward.d;
                }
                const float sampled_cosine = fmaxf(dot(normal, outgoing.d), 0.0f);
                if (sampled_cosine == 0.0f) return true;
                const float brdf_pdf = sampled_cosine / kPi;
                previous_pdf = 0.5f * (brdf_pdf + ground_reflector_pdf(S, K, outgoing));
                path_weight = brdf_pdf / previous_pdf;
            }
        }
        throughput = throughput * (albedo * path_weight);
        if constexpr (G::adjoint) {
            factor(grad, albedo_e);
            grad.prev_param = kNoParam;
        }
        if (depth >= 2u) {
            const float survival = clampf(max3(throughput), 0.05f, 0.95f);
            const bool survived = !(rnd(K, rng) >= survival);
            if constexpr (G::adjoint) {
                if (!grad.pass2) record_roulette(grad, p.iterations, throughput, survival, survived, radiance);
            }
            if (!survived) return true;
            throughput = throughput / survival;
        }
        ray = outgoing;
        previous_vertex = outgoing;
        if constexpr (G::air) {
            p.in_air = inside_air(S, outgoing);
            p.sky_on_escape = sky_lit;
        }
        depth += 1u;
        null_crossings = 0u;
        return false;
    }
}

// One iteration of trace()'s loop (pathtrace.wgsl:1380-1607).
// Returns true when the path has ended. G is the hook set: NoGrad for the
// forward integrator (every hook compiles out), Prb for the adjoint, whose
// first replay records the ring-cap vertex and later Russian roulette and
// whose second scatters derivatives. Hooks never change the path's own
// arithmetic or random draws, so every replay takes the same decisions.
template <bool C, bool L, bool F, class G>
__device__ __forceinline__ bool step(const Scene &S, Counter<C, L, F> K, Path &p, G &grad, Cull cull = kTestAll) {
    Extension e;
    if (!extend(S, K, p, grad, e, cull)) return true;
    if (e.ring.index != kMiss) return ring_vertex(S, K, p, e.ring, grad);
    return surface_vertex(S, K, p, e.hit, e.disc_scale, grad);
}

// The cull masks of the camera rays of 16x16 tile `tile` (kTestAll when the
// frame has none, or for the counting kernel, whose events must be the
// reference algorithm's).
template <bool C>
__device__ __forceinline__ Cull camera_cull(const TraceParams &P, uint32_t tile) {
    if (C || !P.camera_cull) return kTestAll;
    const uint2 m = P.camera_cull[tile];
    return Cull{m.x, m.y};
}

// Stage the body table (and small ring tables) into shared memory.
__device__ __forceinline__ Scene stage_scene(const TraceParams &P, float4 *smem) {
    const uint32_t words = P.s.counts[0] * kBodyVec4;
    for (uint32_t k = threadIdx.x; k < words; k += blockDim.x) smem[k] = P.bodies[k];
    float *staged = reinterpret_cast<float *>(smem + words);
    for (uint32_t k = threadIdx.x; k < P.staged_table_floats; k += blockDim.x) staged[k] = P.tables[k];
    __syncthreads();
    Scene sc;
    sc.p = &P;
    sc.s = &P.s;
    sc.B = smem;
    sc.tables = P.staged_table_floats > 0u ? staged : P.tables;
    return sc;
}

// Floats of dynamic shared memory stage_scene fills.
__device__ __forceinline__ uint32_t trace_smem_floats(const TraceParams &P) {
    return P.s.counts[0] * (uint32_t)kBodyVec4 * 4u + P.staged_table_floats;
}

}  // namespace

}  // namespace sg
