// Per-hit device functions of the radiance loop: texture sampling, surface reconstruction,
// BSDF evaluation/sampling, the HDR environment, the light sampler, secondary-ray offsets
// and camera rays. Each restates the cited CPU-Renderer function with the same operation
// order so that, compiled without FMA contraction, float and double results round as the
// reference's do (transcendentals excepted, see cr_dev_math.cuh).
#pragma once
#include "cr_dev_math.cuh"
#include "cr_internal.h"
#include "cr_traverse.cuh"

namespace crg {

struct F4 { float x, y, z, w; };

// ---- texture sampler (geometry.cpp:68-98, 238-275) ----------------------------------------
CR_D float srgbToLinear(float v) { return v <= 0.04045f ? v / 12.92f : fpow((v + 0.055f) / 1.055f, 2.4f); }  // math.h:61
CR_D double wrappedCoordinate(double value, int32_t wrap) {
    if (wrap == CR_WRAP_CLAMP) return sclamp(value, 0.0, 1.0);
    if (wrap == CR_WRAP_REPEAT) return value - floor(value);
    double result = fmod(value, 2.0);
    if (result < 0) result += 2;
    return result <= 1 ? result : 2 - result;
}
CR_D int wrappedIndex(int64_t index, int size, int32_t wrap) {
    const int64_t n = size;
    if (wrap == CR_WRAP_CLAMP) return static_cast<int>(sclamp(index, int64_t{0}, n - 1));
    const int64_t period = wrap == CR_WRAP_MIRROR ? 2 * n : n;
    index %= period;
    if (index < 0) index += period;
    if (wrap == CR_WRAP_MIRROR && index >= n) index = period - 1 - index;
    return static_cast<int>(index);
}
CR_D F4 interpolate4(F4 a, F4 b, float t) {
    return {a.x * (1 - t) + b.x * t, a.y * (1 - t) + b.y * t, a.z * (1 - t) + b.z * t, a.w * (1 - t) + b.w * t};
}
// slot index: 0 baseColor, 1 metallicRoughness, 2 normal, 3 emissive, 4 transmission.
CR_D const cr_texture_slot& slotOf(const cr_material& m, int k) {
    return k == 0 ? m.base_color_texture : k == 1 ? m.metallic_roughness_texture : k == 2 ? m.normal_texture
         : k == 3 ? m.emissive_texture : m.transmission_texture;
}
CR_D F4 sampleTexture(const DevScene& S, uint32_t material, int k, float2 uv0, float2 uv1, bool srgb, int& err) {
    const cr_material& m = S.materials[material];
    const cr_texture_slot& slot = slotOf(m, k);
    if (slot.texture == -1) return {1, 1, 1, 1};
    const cr_texture tex = S.textures[slot.texture];
    const DevImage im = S.images[tex.image];
    const float2 uv = slot.texcoord == 0 ? uv0 : uv1;
    if (!isfin(uv.x) || !isfin(uv.y)) { err = kErrTextureCoordinates; return {1, 1, 1, 1}; }
    const double2 cs = S.slot_trig[5 * material + k];
    const double c = cs.x, s = cs.y;
    const double x = static_cast<double>(uv.x) * slot.scale[0], y = static_cast<double>(uv.y) * slot.scale[1];
    const double u = wrappedCoordinate(c * x - s * y + slot.offset[0], tex.wrap_s);
    const double v = wrappedCoordinate(s * x + c * y + slot.offset[1], tex.wrap_t);
    auto texel = [&](int64_t ix, int64_t iy) -> F4 {
        const int tx = wrappedIndex(ix, im.width, tex.wrap_s), ty = wrappedIndex(iy, im.height, tex.wrap_t);
        const float4 p = im.pixels[static_cast<size_t>(ty) * static_cast<size_t>(im.width) + static_cast<size_t>(tx)];
        F4 value{p.x, p.y, p.z, p.w};
        if (srgb) { value.x = srgbToLinear(value.x); value.y = srgbToLinear(value.y); value.z = srgbToLinear(value.z); }
        return value;
    };
    if (!tex.linear) return texel(static_cast<int64_t>(floor(u * im.width)), static_cast<int64_t>(floor(v * im.height)));
    const double px = u * im.width - 0.5, py = v * im.height - 0.5;
    const int64_t ix = static_cast<int64_t>(floor(px)), iy = static_cast<int64_t>(floor(py));
    const float fx = static_cast<float>(px - floor(px)), fy = static_cast<float>(py - floor(py));
    return interpolate4(interpolate4(texel(ix, iy), texel(ix + 1, iy), fx),
                        interpolate4(texel(ix, iy + 1), texel(ix + 1, iy + 1), fx), fy);
}
CR_D float2 interpolateUv(const cr_triangle& t, double hu, double hv, int set) {
    const double w = 1.0 - hu - hv;
    return make_float2(static_cast<float>(w * t.v[0].uv[set][0] + hu * t.v[1].uv[set][0] + hv * t.v[2].uv[set][0]),
                       static_cast<float>(w * t.v[0].uv[set][1] + hu * t.v[1].uv[set][1] + hv * t.v[2].uv[set][1]));
}

// Alpha-mask half of Scene::accepts (geometry.cpp:287-290).
CR_D bool accepts_alpha(const DevScene& S, uint32_t tri, double u, double v) {
    const cr_triangle& t = S.tris[tri];
    const cr_material& m = S.materials[t.material];
    if (m.alpha_mode != CR_ALPHA_MASK) return true;
    int err = 0;
    const F4 color = sampleTexture(S, t.material, 0, interpolateUv(t, u, v, 0), interpolateUv(t, u, v, 1), false, err);
    return m.base_color[3] * color.w >= m.alpha_cutoff;
}

// ---- surfaceAt (geometry.cpp:401-459) -----------------------------------------------------
struct Surface {
    V3 position, geometricNormal, normal, tangent, bitangent, positionLow;
    V3 baseColor, emission, attenuationColor;
    float metallic, roughness, transmission, ior, thickness, attenuationDistance;
    uint32_t material;
    bool frontFace, doubleSided;
};

// LEAN: the scene has no textures (every texture slot is -1, so every lookup is exactly
// (1, 1, 1, 1)); the instantiation leaves the texture code out of the kernel.
template <bool LEAN = false>
CR_D Surface surfaceAt(const DevScene& S, V3 rayDir, uint32_t tri, double hu, double hv, int& err) {
    const cr_triangle& t = S.tris[tri];
    const cr_material& material = S.materials[t.material];
    const double w = 1.0 - hu - hv;
    const D3 p = D3(v3(t.v[0].position)) * w + D3(v3(t.v[1].position)) * hu + D3(v3(t.v[2].position)) * hv;
    Surface s;
    s.position = V3{static_cast<float>(p.x), static_cast<float>(p.y), static_cast<float>(p.z)};
    s.positionLow = V3{static_cast<float>(p.x - s.position.x), static_cast<float>(p.y - s.position.y),
                       static_cast<float>(p.z - s.position.z)};
    s.geometricNormal = v3(t.geometric_normal);
    s.frontFace = pdot(D3(rayDir), D3(s.geometricNormal)) < 0;
    s.normal = unit(D3(v3(t.v[0].normal)) * w + D3(v3(t.v[1].normal)) * hu + D3(v3(t.v[2].normal)) * hv, s.geometricNormal);
    if (dot(s.normal, s.geometricNormal) < 0) s.normal = -s.normal;
    auto tangentOf = [](const cr_vertex& v) { return D3(V3{v.tangent[0], v.tangent[1], v.tangent[2]}); };
    s.tangent = orthogonalized(tangentOf(t.v[0]) * w + tangentOf(t.v[1]) * hu + tangentOf(t.v[2]) * hv, s.normal,
                               Frame(s.normal).x);
    float handedness = w * t.v[0].tangent[3] + hu * t.v[1].tangent[3] + hv * t.v[2].tangent[3] < 0 ? -1.0f : 1.0f;
    s.bitangent = cross(s.normal, s.tangent) * handedness;
    float2 uv0 = make_float2(0, 0), uv1 = make_float2(0, 0);
    F4 base{1, 1, 1, 1}, mr{1, 1, 1, 1}, emissive{1, 1, 1, 1}, transmissive{1, 1, 1, 1};
    if constexpr (!LEAN) {
        const bool textured = material.base_color_texture.texture >= 0 || material.metallic_roughness_texture.texture >= 0 ||
                              material.normal_texture.texture >= 0 || material.emissive_texture.texture >= 0 ||
                              material.transmission_texture.texture >= 0;
        if (textured) { uv0 = interpolateUv(t, hu, hv, 0); uv1 = interpolateUv(t, hu, hv, 1); }
        base = sampleTexture(S, t.material, 0, uv0, uv1, true, err);
        mr = sampleTexture(S, t.material, 1, uv0, uv1, false, err);
        emissive = sampleTexture(S, t.material, 3, uv0, uv1, true, err);
        transmissive = sampleTexture(S, t.material, 4, uv0, uv1, false, err);
    }
    s.baseColor = V3{material.base_color[0], material.base_color[1], material.base_color[2]} * V3{base.x, base.y, base.z};
    s.metallic = sclamp(material.metallic * mr.z, 0.0f, 1.0f);
    s.roughness = sclamp(material.roughness * mr.y, 0.0f, 1.0f);
    s.emission = v3(material.emission) * V3{emissive.x, emissive.y, emissive.z};
    s.transmission = sclamp(material.transmission * transmissive.x, 0.0f, 1.0f);
    s.ior = material.ior;
    s.thickness = material.thickness;
    s.attenuationDistance = material.attenuation_distance;
    s.attenuationColor = v3(material.attenuation_color);
    s.material = t.material;
    s.doubleSided = material.double_sided != 0;
    if (!LEAN && material.normal_texture.texture >= 0) {
        const cr_texture_slot& slot = material.normal_texture;
        if (slot.scale[0] != 0 && slot.scale[1] != 0) {
            const double2 cs = S.slot_trig[5 * t.material + 2];
            const D3 tt = D3(s.tangent) * (cs.x / slot.scale[0]) - D3(s.bitangent) * (cs.y / slot.scale[1]);
            s.tangent = orthogonalized(tt, s.normal, s.tangent);
            if ((slot.scale[0] < 0) != (slot.scale[1] < 0)) handedness = -handedness;
            s.bitangent = cross(s.normal, s.tangent) * handedness;
        }
        const F4 texel = sampleTexture(S, t.material, 2, uv0, uv1, false, err);
        const D3 mapped = D3(s.tangent) * ((2.0 * texel.x - 1) * material.normal_scale) +
                          D3(s.bitangent) * ((2.0 * texel.y - 1) * material.normal_scale) +
                          D3(s.normal) * (2.0 * texel.z - 1);
        s.normal = unit(mapped, s.normal);
        if (dot(s.normal, s.geometricNormal) < 0) s.normal = -s.normal;
        s.tangent = orthogonalized(D3(s.tangent), s.normal, Frame(s.normal).x);
        s.bitangent = cross(s.normal, s.tangent) * handedness;
    }
    return s;
}

// ---- BSDF (bsdf.cpp:6-237) ---------------------------------------------------------------
CR_D float fresnelDielectric(float cosine, float etaI, float etaT) {
    if (etaI == etaT) return 0;
    cosine = sclamp(fabsf(cosine), 0.0f, 1.0f);
    const float eta = etaI / etaT;
    const float sinT2 = eta * eta * smax(0.0f, 1 - cosine * cosine);
    if (sinT2 >= 1) return 1;
    const float cosT = sqrtf(1 - sinT2);
    const float ds = etaI * cosine + etaT * cosT, dp = etaT * cosine + etaI * cosT;
    if (ds == 0 || dp == 0) return 1;
    const float rs = (etaI * cosine - etaT * cosT) / ds, rp = (etaT * cosine - etaI * cosT) / dp;
    return 0.5f * (rs * rs + rp * rp);
}
CR_D bool refractDirection(V3 wo, V3 normal, float ratio, V3& wi) {
    const float cosI = dot(wo, normal);
    const float sinT2 = ratio * ratio * smax(0.0f, 1 - cosI * cosI);
    if (sinT2 >= 1) return false;
    wi = normalize(-wo * ratio + normal * (ratio * cosI - sqrtf(1 - sinT2)));
    return true;
}
CR_D V3 absorptionCoefficient(V3 color, float distance) {
    if (!isfin(distance)) return V3{};
    color = vclamp(color, 1e-8f, 1);
    return {-flog(color.x) / distance, -flog(color.y) / distance, -flog(color.z) / distance};
}
CR_D V3 beerLambert(V3 coefficient, float distance) {
    if (distance == kInf) return {coefficient.x > 0 ? 0.0f : 1.0f, coefficient.y > 0 ? 0.0f : 1.0f, coefficient.z > 0 ? 0.0f : 1.0f};
    return vexp(coefficient * (-smax(0.0f, distance)));
}
CR_D float distribution(float alpha, V3 h) {
    if (h.z <= 0) return 0;
    const float a2 = alpha * alpha;
    const float d = (h.x * h.x + h.y * h.y) + a2 * h.z * h.z;
    return a2 / (kPi * d * d);
}
CR_D float smithG1(float alpha, V3 v) {
    const float cos2 = v.z * v.z;
    if (cos2 == 0) return 0;
    return 2 / (1 + sqrtf(1 + alpha * alpha * (v.x * v.x + v.y * v.y) / cos2));
}
CR_D V3 visibleNormal(V3 wo, float alpha, float u, float v) {
    const V3 vh = normalize({alpha * wo.x, alpha * wo.y, wo.z});
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const V3 t1 = lensq > 0 ? V3{-vh.y, vh.x, 0} / sqrtf(lensq) : V3{1, 0, 0};
    const V3 t2 = cross(vh, t1);
    const float r = sqrtf(u), phi = 2 * kPi * v;
    float sp, cp;
    fsincos(phi, sp, cp);
    const float x = r * cp;
    float y = r * sp;
    const float s = 0.5f * (1 + vh.z);
    y = (1 - s) * sqrtf(smax(0.0f, 1 - x * x)) + s * y;
    const V3 nh = t1 * x + t2 * y + vh * sqrtf(smax(0.0f, 1 - x * x - y * y));
    return normalize({alpha * nh.x, alpha * nh.y, smax(0.0f, nh.z)});
}

struct Ctx {
    const Surface& s;
    Frame frame;
    V3 wo;
    float etaI, etaT, eta, alpha, diffuseProbability, deltaTransmissionProbability;
    bool thin, smooth, matched;
    CR_D float fresnel(float cosine) const {
        const float f = fresnelDielectric(cosine, etaI, etaT);
        return thin ? 2 * f / (1 + f) : f;
    }
    CR_D V3 reflection(float f, float cosine) const {
        const float schlick = fpow5(1 - sclamp(fabsf(cosine), 0.0f, 1.0f));
        return V3{(1 - s.metallic) * f} + (s.baseColor + (V3{1} - s.baseColor) * schlick) * s.metallic;
    }
    CR_D V3 transmission(float f) const { return s.baseColor * ((1 - s.metallic) * s.transmission * (1 - f)); }
    CR_D float reflectionProbability(float f, float cosH) const {
        if (matched) return 1;
        const float r = luminance(reflection(f, cosH)), t = luminance(transmission(f));
        return r + t > 0 ? r / (r + t) : 1;
    }
    CR_D float microProbability() const { return smax(0.0f, 1 - diffuseProbability - deltaTransmissionProbability); }
    CR_D Ctx(const Surface& surface, V3 outgoing)
        : s(surface), frame(dot(outgoing, surface.normal) > 0 ? surface.normal : -surface.normal) {
        wo = frame.local(outgoing);
        etaI = s.thickness > 0 && !s.frontFace ? s.ior : 1;
        etaT = s.thickness > 0 && !s.frontFace ? 1 : s.ior;
        eta = etaT / etaI;
        alpha = smax(0.001f, s.roughness * s.roughness);
        diffuseProbability = 0;
        deltaTransmissionProbability = 0;
        thin = s.thickness <= 0 && s.transmission > 0;
        smooth = s.roughness <= 0.001f;
        matched = false;
        if (thin) { etaI = 1; etaT = s.ior; eta = s.ior; }
        matched = fabsf(etaI - etaT) <= sqrtf(kFltEps) * smax(etaI, etaT);
        if (matched) etaI = etaT = eta = 1;
        const float f = fresnel(wo.z);
        const float diffuse = (1 - s.metallic) * (1 - s.transmission) * luminance(s.baseColor) * (1 - f);
        const float transmit = (1 - s.metallic) * s.transmission * (1 - f) * luminance(s.baseColor);
        const float total = diffuse + luminance(reflection(f, wo.z)) + transmit;
        if (total > 0) {
            diffuseProbability = diffuse / total;
            if (matched) deltaTransmissionProbability = transmit / total;
        }
    }
};

struct BsdfEval { V3 value; float pdf; };
struct BsdfSample {
    V3 direction, weight;
    float pdf, eta;
    bool delta, transmitted;
    CR_D bool ok() const { return maxComponent(weight) > 0 && finite3(weight) && finite3(direction); }
};
CR_D BsdfSample emptySample() { BsdfSample b; b.direction = V3{}; b.weight = V3{}; b.pdf = 0; b.eta = 1; b.delta = false; b.transmitted = false; return b; }

CR_D BsdfEval evalLocal(const Ctx& c, V3 wi) {
    BsdfEval result{V3{}, 0};
    const float no = c.wo.z, ni = fabsf(wi.z);
    if (no <= 1e-7f || ni <= 1e-7f) return result;
    const bool reflection = wi.z > 0;
    if (!reflection && (c.matched || c.thin)) return result;
    if (reflection) {
        const float diffuse = (1 - c.s.metallic) * (1 - c.s.transmission) * (1 - c.fresnel(no)) * (1 - c.fresnel(ni));
        result.value = c.s.baseColor * (diffuse / kPi);
        result.pdf = c.diffuseProbability * ni / kPi;
    }
    if (c.smooth) return result;
    V3 h = normalize(reflection ? c.wo + wi : c.wo + wi * c.eta);
    if (h.z < 0) h = -h;
    const float oh = dot(c.wo, h), ih = dot(wi, h);
    if (oh <= 0 || (reflection ? ih <= 0 : ih >= 0)) return result;
    const float f = c.fresnel(oh), pr = c.reflectionProbability(f, oh);
    const float d = distribution(c.alpha, h), g1 = smithG1(c.alpha, c.wo), g = g1 * smithG1(c.alpha, wi);
    const float pdfH = d * g1 * oh / no;
    if (reflection) {
        result.value = result.value + c.reflection(f, oh) * (d * g / (4 * no * ni));
        result.pdf += c.microProbability() * pr * pdfH / (4 * oh);
    } else {
        const float denom = oh + c.eta * ih, denom2 = denom * denom;
        if (denom2 < 1e-20f) return BsdfEval{V3{}, 0};
        result.value = c.transmission(f) * (d * g * fabsf(oh * ih) / (no * ni * denom2));
        result.pdf = c.microProbability() * (1 - pr) * pdfH * c.eta * c.eta * fabsf(ih) / denom2;
    }
    return result;
}
CR_D bool correctGeometricSide(const Surface& s, V3 wo, V3 wi, bool transmitted) {
    const float d = dot(wo, s.geometricNormal) * dot(wi, s.geometricNormal);
    return transmitted ? d < 0 : d > 0;
}
CR_D BsdfEval evaluateBsdf(const Surface& s, V3 wo, V3 wi) {
    const Ctx c(s, wo);
    const V3 local = c.frame.local(wi);
    if (!correctGeometricSide(s, wo, wi, local.z < 0)) return BsdfEval{V3{}, 0};
    return evalLocal(c, local);
}
CR_D BsdfSample sampleBsdf(const Surface& s, V3 wo, Rng& rng) {
    const Ctx c(s, wo);
    BsdfSample out = emptySample();
    if (c.wo.z <= 1e-7f) return out;
    V3 wi;
    const float lobe = rng.uniform();
    if (lobe < c.diffuseProbability) {
        const float u = rng.uniform(), phi = 2 * kPi * rng.uniform();
        float sp, cp;
        fsincos(phi, sp, cp);
        wi = V3{sqrtf(u) * cp, sqrtf(u) * sp, sqrtf(1 - u)};
    } else if (lobe < c.diffuseProbability + c.deltaTransmissionProbability) {
        out.direction = -wo; out.delta = true; out.transmitted = true; out.pdf = c.deltaTransmissionProbability;
        out.weight = s.baseColor * ((1 - s.metallic) * s.transmission / out.pdf);
        return correctGeometricSide(s, wo, out.direction, true) ? out : emptySample();
    } else {
        const float u = rng.uniform(), v = rng.uniform();
        const V3 h = c.smooth ? V3{0, 0, 1} : visibleNormal(c.wo, c.alpha, u, v);
        const float oh = dot(c.wo, h), f = c.fresnel(oh), pr = c.reflectionProbability(f, oh);
        const bool reflection = rng.uniform() < pr;
        if (reflection) wi = reflect(-c.wo, h);
        else if (c.thin) wi = -c.wo;
        else if (!refractDirection(c.wo, h, 1 / c.eta, wi)) return out;
        if ((reflection && wi.z <= 0) || (!reflection && wi.z >= 0)) return out;
        out.transmitted = !reflection;
        out.eta = out.transmitted && !c.thin ? c.eta : 1;
        if (c.smooth || (!reflection && c.thin)) {
            out.delta = true;
            out.direction = normalize(c.frame.world(wi));
            if (!correctGeometricSide(s, wo, out.direction, out.transmitted)) return emptySample();
            const float prob = c.microProbability() * (reflection ? pr : 1 - pr);
            if (prob <= 0) return emptySample();
            out.pdf = prob;
            out.weight = (reflection ? c.reflection(f, oh) : c.transmission(f) / (out.eta * out.eta)) / prob;
            return out;
        }
    }
    out.direction = normalize(c.frame.world(wi));
    wi = c.frame.local(out.direction);
    if ((wi.z < 0) != out.transmitted || !correctGeometricSide(s, wo, out.direction, out.transmitted)) return emptySample();
    const BsdfEval e = evalLocal(c, wi);
    if (e.pdf <= 0 || !isfin(e.pdf)) return emptySample();
    out.pdf = e.pdf;
    out.weight = e.value * (fabsf(wi.z) / e.pdf);
    return out;
}

// sampleBsdf for a kTriNeeNull surface: smooth (roughness <= 0.001 with no texture that could
// change it), and metallic exactly 1 or transmission exactly 1 (no texture that could change
// it). Its diffuse weight (1 - metallic) * (1 - transmission) * ... is then 0 (or NaN, which
// leaves the total not above 0 and every probability 0), so the diffuse lobe is never drawn,
// and the microfacet lobe is smooth, so it returns its delta sample before any evaluation.
// What remains is sampleBsdf's own arithmetic on those two branches, drawing the same numbers
// (u and v of the microfacet lobe are drawn and unused, as there).
CR_D BsdfSample sampleSmooth(const Surface& s, V3 wo, Rng& rng) {
    const Ctx c(s, wo);
    BsdfSample out = emptySample();
    if (c.wo.z <= 1e-7f) return out;
    const float lobe = rng.uniform();
    if (lobe < c.diffuseProbability + c.deltaTransmissionProbability) {
        out.direction = -wo; out.delta = true; out.transmitted = true; out.pdf = c.deltaTransmissionProbability;
        out.weight = s.baseColor * ((1 - s.metallic) * s.transmission / out.pdf);
        return correctGeometricSide(s, wo, out.direction, true) ? out : emptySample();
    }
    rng.uniform();
    rng.uniform();
    const V3 h{0, 0, 1};
    const float oh = dot(c.wo, h), f = c.fresnel(oh), pr = c.reflectionProbability(f, oh);
    const bool reflection = rng.uniform() < pr;
    V3 wi;
    if (reflection) wi = reflect(-c.wo, h);
    else if (c.thin) wi = -c.wo;
    else if (!refractDirection(c.wo, h, 1 / c.eta, wi)) return out;
    if ((reflection && wi.z <= 0) || (!reflection && wi.z >= 0)) return out;
    out.transmitted = !reflection;
    out.eta = out.transmitted && !c.thin ? c.eta : 1;
    out.delta = true;
    out.direction = normalize(c.frame.world(wi));
    if (!correctGeometricSide(s, wo, out.direction, out.transmitted)) return emptySample();
    const float prob = c.microProbability() * (reflection ? pr : 1 - pr);
    if (prob <= 0) return emptySample();
    out.pdf = prob;
    out.weight = (reflection ? c.reflection(f, oh) : c.transmission(f) / (out.eta * out.eta)) / prob;
    return out;
}

// ---- GGX conductor (the bsdf.cpp BSDF at metallic exactly 1, transmission exactly 0) -----------
// A material with metallic 1, transmission 0 and no texture that could change either (the
// kTriConductor surfaces) has, in the BSDF above: diffuse and transmission weights
// (1 - metallic) * ... = 0 for finite factors, so the diffuse lobe's probability and the delta
// transmission probability are 0, the micro-facet lobe's probability 1 - 0 - 0 = 1 and the
// reflection probability r / (r + 0) = 1; the reflection colour (1 - metallic) * F + C * 1 = C.
// The functions below are that BSDF with the exact zeros left out: the same values, pdfs and
// random draws (the lobe and reflection draws are consumed and cannot change the outcome), so
// the conductor shading kernel renders what the generic one renders, with far less code.
struct CondCtx {
    const Surface& s;
    Frame frame;
    V3 wo;
    float alpha;
    bool smooth;
    CR_D CondCtx(const Surface& surface, V3 outgoing)
        : s(surface), frame(dot(outgoing, surface.normal) > 0 ? surface.normal : -surface.normal) {
        wo = frame.local(outgoing);
        alpha = smax(0.001f, s.roughness * s.roughness);
        smooth = s.roughness <= 0.001f;
    }
    CR_D V3 reflection(float cosine) const {
        const float schlick = fpow5(1 - sclamp(fabsf(cosine), 0.0f, 1.0f));
        return s.baseColor + (V3{1} - s.baseColor) * schlick;
    }
};
CR_D BsdfEval evalConductor(const CondCtx& c, V3 wi) {
    const BsdfEval zero{V3{}, 0};
    const float no = c.wo.z, ni = fabsf(wi.z);
    if (no <= 1e-7f || ni <= 1e-7f) return zero;
    if (!(wi.z > 0) || c.smooth) return zero;  // transmission is zero; a smooth lobe is a delta
    V3 h = normalize(c.wo + wi);
    if (h.z < 0) h = -h;
    const float oh = dot(c.wo, h), ih = dot(wi, h);
    if (oh <= 0 || ih <= 0) return zero;
    const float d = distribution(c.alpha, h), g1 = smithG1(c.alpha, c.wo), g = g1 * smithG1(c.alpha, wi);
    const float pdfH = d * g1 * oh / no;
    return BsdfEval{c.reflection(oh) * (d * g / (4 * no * ni)), pdfH / (4 * oh)};
}
CR_D BsdfEval evaluateConductor(const Surface& s, V3 wo, V3 wi) {
    const CondCtx c(s, wo);
    const V3 local = c.frame.local(wi);
    if (!correctGeometricSide(s, wo, wi, local.z < 0)) return BsdfEval{V3{}, 0};
    return evalConductor(c, local);
}
CR_D BsdfSample sampleConductor(const Surface& s, V3 wo, Rng& rng) {
    const CondCtx c(s, wo);
    BsdfSample out = emptySample();
    if (c.wo.z <= 1e-7f) return out;
    rng.uniform();  // the lobe draw: the micro-facet lobe has probability 1
    const float u = rng.uniform(), v = rng.uniform();
    const V3 h = c.smooth ? V3{0, 0, 1} : visibleNormal(c.wo, c.alpha, u, v);
    const float oh = dot(c.wo, h);
    rng.uniform();  // the reflection draw: reflection has probability 1
    V3 wi = reflect(-c.wo, h);
    if (wi.z <= 0) return out;
    out.transmitted = false;
    out.eta = 1;
    if (c.smooth) {
        out.delta = true;
        out.direction = normalize(c.frame.world(wi));
        if (!correctGeometricSide(s, wo, out.direction, false)) return emptySample();
        out.pdf = 1;
        out.weight = c.reflection(oh);
        return out;
    }
    out.direction = normalize(c.frame.world(wi));
    wi = c.frame.local(out.direction);
    if (wi.z < 0 || !correctGeometricSide(s, wo, out.direction, false)) return emptySample();
    const BsdfEval e = evalConductor(c, wi);
    if (e.pdf <= 0 || !isfin(e.pdf)) return emptySample();
    out.pdf = e.pdf;
    out.weight = e.value * (fabsf(wi.z) / e.pdf);
    return out;
}

// ---- environment (render.cpp:10-94) ----------------------------------------------------------
CR_D float2 envUv(const DevScene& S, V3 d) {
    float u = (fatan2(d.z, d.x) - S.env_rotation) / (2 * kPi) + 0.5f;
    u -= floorf(u);
    return make_float2(u, facos(sclamp(d.y, -1.0f, 1.0f)) / kPi);
}
CR_D V3 envRadiance(const DevScene& S, V3 d) {
    if (!S.env_has_image) return v3(S.env_constant);
    const float2 coord = envUv(S, d);
    const int W = S.env_width, H = S.env_height;
    const float px = coord.x * static_cast<float>(W) - 0.5f, py = coord.y * static_cast<float>(H) - 0.5f;
    const int x = static_cast<int>(floorf(px)), y = static_cast<int>(floorf(py));
    const float tx = px - static_cast<float>(x), ty = py - static_cast<float>(y);
    auto texel = [&](int ix, int iy) {
        ix = (ix % W + W) % W;
        iy = sclamp(iy, 0, H - 1);
        const float4 p = __ldg(S.env_pixels + static_cast<size_t>(iy) * W + ix);
        return V3{p.x, p.y, p.z};
    };
    return mix(mix(texel(x, y), texel(x + 1, y), tx), mix(texel(x, y + 1), texel(x + 1, y + 1), tx), ty) * S.env_intensity;
}
CR_D float envPdf(const DevScene& S, V3 d) {
    if (!S.env_has_image) return 1 / (4 * kPi);
    const float2 coord = envUv(S, d);
    const int x = smin(static_cast<int>(coord.x * static_cast<float>(S.env_width)), S.env_width - 1);
    const int y = smin(static_cast<int>(coord.y * static_cast<float>(S.env_height)), S.env_height - 1);
    return __ldg(S.env_pdf + static_cast<size_t>(y) * S.env_width + x);
}
// std::upper_bound over the FP64 CDF, first narrowed by a bracket table: env_coarse[j] is
// the upper bound of j*weightSum/K (K = env_coarse_count). A pick in bracket j has its
// answer in [env_coarse[j], env_coarse[j+1]]; taking one extra bracket on each side absorbs
// any rounding in locating j, so the search below returns exactly the full search's index.
CR_D uint32_t envUpperBound(const DevScene& S, double pick) {
    const uint64_t n = static_cast<uint64_t>(S.env_width) * S.env_height;
    uint64_t lo = 0, hi = n;
    const int64_t K = S.env_coarse_count;
    if (K) {
        int64_t j = static_cast<int64_t>(floor(pick / S.env_weight_sum * static_cast<double>(K)));
        j = j < 0 ? 0 : (j > K - 1 ? K - 1 : j);
        lo = j >= 1 ? __ldg(S.env_coarse + (j - 1)) : 0;
        hi = j + 2 <= K - 1 ? __ldg(S.env_coarse + (j + 2)) : n;
    }
    uint64_t count = hi - lo;
    while (count > 0) {
        const uint64_t step = count / 2;
        const uint64_t it = lo + step;
        if (!(pick < __ldg(S.env_cdf + it))) { lo = it + 1; count -= step + 1; }
        else count = step;
    }
    return static_cast<uint32_t>(lo);
}
// The texel an environment-image sample takes (Environment::sample's first step,
// render.cpp:73-75, or the alias table).
CR_D uint64_t envPickTexel(const DevScene& S, Rng& rng, bool alias) {
    const uint64_t n = static_cast<uint64_t>(S.env_width) * S.env_height;
    uint64_t index;
    if (alias && S.alias_threshold) {
        // Walker's alias method (Walker 1977; Vose 1991). Two draws form a 48-bit uniform x;
        // x*n = col*2^48 + r gives the column and a 48-bit residual that chooses between the
        // column and its alias (the host set the thresholds so that every texel's probability
        // is an exact count over 2^48, and env_pdf holds those densities). A different stream
        // from the CDF search: used only when alias sampling is requested.
        const uint64_t a = rng.next() >> 8, b = rng.next() >> 8;
        const uint64_t xs = ((a << 24) | b) << 16;
        const uint64_t col = __umul64hi(xs, n);        // < n: x < 2^48
        const uint64_t r = (xs * n) >> 16;            // (x*n) mod 2^48
        index = r < __ldg(S.alias_threshold + col) ? col : __ldg(S.alias_index + col);
    } else {
        const double pick = rng.uniform() * S.env_weight_sum;
        index = envUpperBound(S, pick);
        if (index > n - 1) index = n - 1;
    }
    return index;
}
CR_D V3 envSample(const DevScene& S, Rng& rng, float& density, bool alias) {
    if (!S.env_has_image) {
        const float y = 1 - 2 * rng.uniform(), phi = 2 * kPi * rng.uniform(), r = sqrtf(smax(0.0f, 1 - y * y));
        density = 1 / (4 * kPi);
        float sp, cp;
        fsincos(phi, sp, cp);
        return {r * cp, y, r * sp};
    }
    const uint64_t index = envPickTexel(S, rng, alias);
    const int W = S.env_width, H = S.env_height;
    const int x = static_cast<int>(index % W), y = static_cast<int>(index / W);
    const float u = (static_cast<float>(x) + rng.uniform()) / static_cast<float>(W);
    const float c0 = __ldg(S.env_row_cos + y), c1 = __ldg(S.env_row_cos + y + 1);
    const float cosTheta = c0 + (c1 - c0) * rng.uniform(), sinTheta = sqrtf(smax(0.0f, 1 - cosTheta * cosTheta));
    const float phi = (u - 0.5f) * 2 * kPi + S.env_rotation;
    density = __ldg(S.env_pdf + index);
    float sp, cp;
    fsincos(phi, sp, cp);
    return {sinTheta * cp, cosTheta, sinTheta * sp};
}

// ---- light sampler (render.cpp:113-229) --------------------------------------------------------
struct LightSample {
    V3 direction, radiance, target, targetNormal;
    float distance, pdf;
    bool delta;
};
CR_D LightSample emptyLight() {
    LightSample l; l.direction = l.radiance = l.target = l.targetNormal = V3{}; l.distance = kInf; l.pdf = 0; l.delta = false; return l;
}
CR_D float environmentPdf(const DevScene& S, V3 direction) { return S.env_probability * envPdf(S, direction); }
CR_D float trianglePdf(const DevScene& S, uint32_t index, V3 from, V3 point) {
    const cr_triangle& t = S.tris[index];
    const V3 dir = point - from;
    const float len2 = lengthSquared(dir), cosine = fabsf(dot(v3(t.geometric_normal), normalize(dir)));
    return cosine > 1e-8f ? __ldg(S.tri_light_probability + index) * len2 / (t.area * cosine) : 0;
}
// LEAN: besides having no textures, the scene has no punctual lights and no alpha masks.
template <bool LEAN = false>
CR_D LightSample sampleLight(const DevScene& S, V3 from, Rng& rng, bool alias, int& err) {
    LightSample out = emptyLight();
    if (S.light_entry_count == 0) return out;
    const double u = rng.uniform();
    // std::lower_bound(entries, u, e.cdf < u)
    uint32_t lo = 0, count = S.light_entry_count;
    while (count > 0) {
        const uint32_t step = count / 2, it = lo + step;
        if (S.light_entries[it].cdf < u) { lo = it + 1; count -= step + 1; } else count = step;
    }
    const LightEntry e = S.light_entries[lo == S.light_entry_count ? S.light_entry_count - 1 : lo];
    if (e.type == kLightEnvironment) {
        out.direction = envSample(S, rng, out.pdf, alias);
        out.pdf *= e.probability;
        out.radiance = envRadiance(S, out.direction);
        return out;
    }
    if (!LEAN && e.type == kLightPunctual) {
        const DevPunctual& l = S.punctual[e.index];
        out.delta = true; out.pdf = e.probability;
        float attenuation = 1;
        if (l.type == CR_LIGHT_DIRECTIONAL) out.direction = -v3(l.direction);
        else {
            const V3 delta = v3(l.position) - from;
            const float r2 = lengthSquared(delta);
            if (r2 < 1e-12f) return emptyLight();
            out.distance = sqrtf(r2); out.direction = delta / out.distance; out.target = v3(l.position);
            attenuation = 1 / r2;
            if (isfin(l.range)) {
                const float q = out.distance / l.range;
                attenuation *= smax(0.0f, 1 - q * q * q * q);
            }
            if (l.type == CR_LIGHT_SPOT) {
                const float cosAngle = dot(v3(l.direction), -out.direction), outer = l.cos_outer, inner = l.cos_inner;
                const float falloff = sclamp((cosAngle - outer) / smax(1e-7f, inner - outer), 0.0f, 1.0f);
                attenuation *= falloff * falloff;
            }
        }
        out.radiance = v3(l.color) * (l.intensity * attenuation);
        return out;
    }
    const cr_triangle& t = S.tris[e.index];
    const float r = sqrtf(rng.uniform()), u1 = 1 - r, u2 = r * rng.uniform(), u0 = 1 - u1 - u2;
    out.target = v3(t.v[0].position) * u0 + v3(t.v[1].position) * u1 + v3(t.v[2].position) * u2;
    out.targetNormal = v3(t.geometric_normal);
    const V3 delta = out.target - from;
    out.distance = length(delta);
    if (out.distance < 1e-7f) return emptyLight();
    out.direction = delta / out.distance;
    // Scene::accepts on Ray{from, direction} with Hit{distance, u1, u2}
    const uint32_t flags = __float_as_uint(__ldg(S.tri_ng + e.index).w);
    if ((flags & kTriCull) && !accepts_cull(S, e.index, out.direction)) return emptyLight();
    if (!LEAN && (flags & kTriAlphaMask) && !accepts_alpha(S, e.index, u1, u2)) return emptyLight();
    const Surface s = surfaceAt<LEAN>(S, out.direction, e.index, u1, u2, err);
    if (!s.frontFace && !s.doubleSided) return emptyLight();
    out.radiance = s.emission;
    out.pdf = trianglePdf(S, e.index, from, out.target);
    return out;
}

// The random draws sampleLight consumes, without its arithmetic: for a surface whose BSDF is
// zero in every direction the light sample cannot contribute (render.cpp:271-272), but its
// draws still advance the stream (1 selection draw; environment image 3, constant
// environment 2, alias table 4, triangle 2, punctual 0).
CR_D void skipLight(const DevScene& S, Rng& rng, bool alias) {
    if (S.light_entry_count == 0) return;
    const double u = rng.uniform();
    uint32_t lo = 0, count = S.light_entry_count;
    while (count > 0) {
        const uint32_t step = count / 2, it = lo + step;
        if (S.light_entries[it].cdf < u) { lo = it + 1; count -= step + 1; } else count = step;
    }
    const uint32_t type = S.light_entries[lo == S.light_entry_count ? S.light_entry_count - 1 : lo].type;
    int draws = 0;
    if (type == kLightEnvironment) draws = !S.env_has_image ? 2 : (alias && S.alias_threshold ? 4 : 3);
    else if (type == kLightTriangle) draws = 2;
    for (int k = 0; k < draws; ++k) rng.next();
}

// ---- offsetRay (geometry.cpp:186-209) ------------------------------------------------------------
// Returns false with err set where the reference throws (invalid_argument / overflow_error).
CR_D bool offsetRay(V3 position, V3 geometricNormal, V3 direction, float maxDistance, TRay& out, int& err) {
    if (!finite3(position) || !finite3(geometricNormal) || !finite3(direction) || !nonzero(geometricNormal) ||
        !nonzero(direction) || isnan(maxDistance) || maxDistance < 0) { err = kErrInvalidSecondaryRay; return false; }
    direction = unit(direction);
    V3 n = unit(geometricNormal);
    if (pdot(D3(n), D3(direction)) < 0) n = -n;
    const double scale = smax3(fabs(static_cast<double>(position.x)), fabs(static_cast<double>(position.y)),
                               fabs(static_cast<double>(position.z)));
    const double distance = (4 * kFltEps) * scale;
    float o[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        o[axis] = static_cast<float>(static_cast<double>(position[axis]) + distance * n[axis]);
        if (n[axis] != 0) o[axis] = n[axis] > 0 ? next_up(o[axis]) : next_down(o[axis]);
    }
    const V3 origin{o[0], o[1], o[2]};
    if (!finite3(origin)) { err = kErrOffsetOverflow; return false; }
    float limit = maxDistance;
    if (isfin(limit)) {
        const double advance = pdot(D3(origin) - D3(position), D3(direction));
        limit = static_cast<float>(smax(0.0, static_cast<double>(limit) - advance));
        limit = next_toward_zero(limit);
    }
    out.o = origin; out.d = direction; out.tmin = 0; out.tmax = limit; out.olow = V3{};
    return true;
}

// ---- Camera::generate per ray (geometry.cpp:225-233); the basis is set up on the host --------------
CR_D bool cameraRay(const DevCamera& C, int width, int height, float pixelX, float pixelY, TRay& out) {
    const double x = (2 * static_cast<double>(pixelX) / width - 1) * C.ratio * C.halfHeight;
    const double y = (1 - 2 * static_cast<double>(pixelY) / height) * C.halfHeight;
    const V3 f = v3(C.f), r = v3(C.r), u = v3(C.u);
    const V3 direction = unit(D3(f) + D3(r) * x + D3(u) * y);
    const double projection = pdot(D3(direction), D3(f));
    const double nearT = C.nearClip / projection;
    if (!(projection > 0) || !isfin(nearT) || nearT > static_cast<double>(kFltMax)) return false;
    out.o = v3(C.position); out.d = direction;
    out.tmin = static_cast<float>(nearT);
    out.tmax = static_cast<float>(C.farClip / projection);
    out.olow = V3{};
    return true;
}

}  // namespace crg
