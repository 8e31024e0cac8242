// bsdf.cuh - the serving integrator's materials, an OpenPBR subset (host + device code).
//
// A material (cwp_material, 64 B) is a fixed mix of three bases, weighted metal = metallic, glass =
// (1 - metallic) transmission, gloss = (1 - metallic)(1 - transmission):
//   metal  a rough conductor whose reflectance is the F82-tint Fresnel curve of (base colour, specular colour),
//          scaled by the specular weight;
//   glass  a rough dielectric interface that reflects and refracts (exact Fresnel), refraction tinted by the base colour;
//   gloss  an opaque dielectric: a GGX specular layer (specular weight, IOR) over a Lambertian base colour.
// All three share one GGX microfacet distribution with alpha = roughness^2; alpha below kSmoothAlpha is a smooth
// surface (a Dirac lobe, sampled but never evaluated).
//
// What an image depends on - which lobes exist, their weights, how a sample picks a base and spends the random
// numbers (u, u1, u2, and ux1, ux2 for the gloss base's albedo estimate), the delta conventions - is the reference's
// (render/bsdf.h), so that both integrators render the same images. The formulas are written here from the papers:
//   GGX normal distribution, the generalised half vector of refraction and its Jacobian, and the exact unpolarised
//     Fresnel reflectance in its g-form: Walter, Marschner, Li, Torrance, EGSR 2007 (eqs. 13-17, 21-22, 33)
//   height-correlated Smith masking-shadowing, G2 = 1 / (1 + Lambda(o) + Lambda(i)), and the distribution of visible
//     normals D_wo(m) = G1(wo) max(0, wo.m) D(m) / wo.z: Heitz, JCGT 2014
//   sampling the visible normals with spherical caps: Dupuy & Benyoub, HPG 2023
//   the conductor's F82-tint Fresnel: Kutz, Hasan, Edmondson 2021, as specified by OpenPBR 1.0
//   the bump-terminator shadowing of the diffuse base: Chiang, Li, Burley, SIGGRAPH 2019 talk
//   the power heuristic: Veach 1997
// Transmission keeps the energy convention: a lossless smooth interface passes a throughput of 1 - F both ways (no
// eta^2 radiance scaling).
// Conventions: local frame with z = the shading normal, wo.z > 0 (towards the viewer). bsdf_eval returns f and the
// solid-angle pdf of the non-delta lobes; bsdf_sample returns wi, weight = f |cos| / pdf and pdf (0 = a delta sample).
#pragma once
#include "cwp_b200.h"
#include "vecmath.h"

namespace cwpb {

#define CWPB_PI 3.14159265f
static constexpr float kSmoothAlpha = 1e-3f;

CWPB_HD float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }   // Rec. 709 weights
CWPB_HD float3 mat_v3(const float* a) { return f3(a[0], a[1], a[2]); }
CWPB_HD float sat(float x) { return fminf(fmaxf(x, 0.f), 1.f); }
CWPB_HD float3 reflect_about(float3 w, float3 m, float wm) { return m * (2.f * wm) - w; }

struct BsdfValue { float3 f; float pdf; };

// ---- the isotropic GGX microfacet model ----
struct Ggx {
    float alpha, a2;
    bool smooth;
    CWPB_HD explicit Ggx(float roughness) : alpha(roughness * roughness), a2(alpha * alpha), smooth(alpha < kSmoothAlpha) {}
    // D(m) = a^2 / (pi ((a^2 - 1) cos^2 + 1)^2) for cos > 0
    CWPB_HD float D(float cosM) const {
        if (!(cosM > 0.f)) return 0.f;
        const float t = (a2 - 1.f) * (cosM * cosM) + 1.f;
        return a2 / (CWPB_PI * t * t);
    }
    // Smith's Lambda: (sqrt(1 + a^2 tan^2) - 1) / 2, unbounded at grazing
    CWPB_HD float Lambda(float cosW) const {
        const float c2 = cosW * cosW;
        if (c2 < 1e-12f) return 1e12f;
        const float tan2 = (1.f - c2) / c2;
        return 0.5f * (sqrtf(1.f + a2 * tan2) - 1.f);
    }
    CWPB_HD float G1(float cosW) const { return 1.f / (1.f + Lambda(cosW)); }
    CWPB_HD float G2(float cosO, float cosI) const { return 1.f / (1.f + Lambda(cosO) + Lambda(cosI)); }
    // density of the normals visible from wo
    CWPB_HD float visible_pdf(float3 wo, float3 m) const {
        const float wm = dot(wo, m);
        if (wm <= 0.f || m.z <= 0.f) return 0.f;
        return G1(wo.z) * wm * D(m.z) / wo.z;
    }
    // a visible normal: wo stretched to the alpha = 1 configuration, a uniform point on the spherical cap of the unit
    // sphere below the stretched direction, offset by it, then unstretched (Dupuy & Benyoub)
    CWPB_HD float3 sample_visible(float3 wo, float u1, float u2) const {
        const float3 s = normalize(f3(alpha * wo.x, alpha * wo.y, wo.z));
        const float z = (1.f - u2) * (1.f + s.z) - s.z;
        const float r = sqrtf(sat(1.f - z * z)), phi = CWPB_TWO_PI * u1;
        const float3 h = f3(r * cosf(phi) + s.x, r * sinf(phi) + s.y, z + s.z);
        return normalize(f3(alpha * h.x, alpha * h.y, fmaxf(h.z, 0.f)));
    }
};

// ---- Fresnel reflectance ----
// exact unpolarised reflectance of a dielectric interface at |cos| = c, eta = n(transmitted side) / n(incident side):
// with g^2 = eta^2 - 1 + c^2 (negative: total internal reflection),
// F = 1/2 ((g - c) / (g + c))^2 (1 + ((c (g + c) - 1) / (c (g - c) + 1))^2)
CWPB_HD float fresnel_exact(float c, float eta) {
    const float g2 = eta * eta - 1.f + c * c;
    if (g2 <= 0.f) return 1.f;
    const float g = sqrtf(g2);
    const float p = (g - c) / (g + c), q = (c * (g + c) - 1.f) / (c * (g - c) + 1.f);
    return 0.5f * p * p * (1.f + q * q);
}
// F82-tint conductor reflectance: Schlick's curve S(mu) = F0 + (1 - F0)(1 - mu)^5 lowered by b mu (1 - mu)^6, where
// b makes the curve equal tint x S at mu = 1/7; clamped to [0, 1] per channel
struct F82Curve {
    float q5, lower;   // (1 - mu)^5 and mu (1 - mu)^6 / (mu_b (1 - mu_b)^6) at this mu
    static constexpr float muB = 1.f / 7.f, qB = 1.f - muB, qB5 = qB * qB * qB * qB * qB;
    CWPB_HD explicit F82Curve(float mu) {
        mu = sat(mu);
        const float q = 1.f - mu;
        q5 = (q * q) * (q * q) * q;
        lower = mu * q5 * q * (1.f / (muB * qB5 * qB));
    }
    CWPB_HD float channel(float f0, float tint) const {
        const float schlick = f0 + (1.f - f0) * q5, schlickB = f0 + (1.f - f0) * qB5;
        return sat(schlick - schlickB * (1.f - tint) * lower);
    }
};
CWPB_HD float3 fresnel_conductor(float3 F0, float3 tint, float mu) {
    const F82Curve c(mu);
    return f3(c.channel(F0.x, tint.x), c.channel(F0.y, tint.y), c.channel(F0.z, tint.z));
}

// ---- bump-terminator shadowing of the diffuse base ----
// nr = the unperturbed normal in the frame of the mapped shading normal; g = (nr . wi) / (wi.z nr.z) is the ratio
// of the two cosines; the smooth step g (1 + g (1 - g)) on [0, 1), 1 above, 0 below. nr = +z switches it off.
CWPB_HD float terminator_shadowing(float3 nr, float3 wi) {
    if (nr.z >= 1.f) return 1.f;
    const float g = dot(nr, wi) / (wi.z * nr.z);
    return g >= 1.f ? 1.f : (g < 0.f ? 0.f : g * (1.f + g * (1.f - g)));
}

// ---- one shading vertex: the three bases of a material for one outgoing direction ----
struct PbrVertex {
    const cwp_material& m;
    Ggx ggx;
    float wMetal, wGlass, wGloss;   // base weights
    float eta;                      // relative IOR of the glass base at this side
    // gloss base: Fresnel at the normal (times the specular weight), probability of sampling its specular layer and
    // the diffuse scale kd; nr for the terminator term
    float glossF, glossPSpec, glossKd;
    float3 nr;

    CWPB_HD PbrVertex(const cwp_material& mat, float3 wo, float etaRel, int gdEnergy, float ux1, float ux2, float3 nrLocal)
        : m(mat), ggx(mat.roughness), eta(etaRel), glossF(0.f), glossPSpec(0.f), glossKd(1.f), nr(nrLocal) {
        wMetal = m.metallic;
        wGlass = (1.f - m.metallic) * m.transmission;
        wGloss = (1.f - m.metallic) * (1.f - m.transmission);
        if (wGloss > 0.f) {
            const float ws = m.specular_weight;
            if (ws > 0.f) glossF = ws * fresnel_exact(wo.z, m.ior);
            const float diffuse = (1.f - glossF) * luminance(mat_v3(m.base_color));
            glossPSpec = glossF + diffuse > 0.f ? glossF / (glossF + diffuse) : 0.f;
            float spec = glossF;   // the specular layer's albedo: F at the normal, or one visible-normal estimate of it
            if (gdEnergy && ws > 0.f && !ggx.smooth) {
                const float3 mm = ggx.sample_visible(wo, ux1, ux2);
                const float wm = dot(wo, mm);
                const float3 wr = reflect_about(wo, mm, wm);
                spec = (wm > 0.f && wr.z > 0.f) ? ws * fresnel_exact(wm, m.ior) * ggx.G2(wo.z, wr.z) / ggx.G1(wo.z) : 0.f;
            }
            glossKd = fmaxf(1.f - spec, 0.f);
        }
    }

    // every non-delta lobe at (wo, wi): the material's f and pdf; with base >= 0 also that base's own (unweighted)
    // pdf in *ownPdf, from the same terms
    CWPB_HD BsdfValue eval(float3 wo, float3 wi, int base = -1, float* ownPdf = nullptr) const {
        BsdfValue r{ f3(0.f, 0.f, 0.f), 0.f };
        float o = 0.f;
        auto add = [&](int b, float weight, float3 f, float pdf) {
            r.f = r.f + f * weight; r.pdf += weight * pdf;
            if (b == base) o = pdf;
        };
        if (wi.z > 0.f) {
            // reflection: the terms every reflecting lobe shares for the half vector of (wo, wi)
            const float3 h = normalize(wo + wi);
            const float wh = dot(wo, h);
            const bool rough = !ggx.smooth && wh > 0.f;
            float micro = 0.f, pdfH = 0.f;   // D G2 / (4 wo.z wi.z) and the reflection pdf of the visible normals
            if (rough) { micro = ggx.D(h.z) * ggx.G2(wo.z, wi.z) / (4.f * wo.z * wi.z); pdfH = ggx.visible_pdf(wo, h) / (4.f * wh); }
            if (wMetal > 0.f && rough) add(0, wMetal, fresnel_conductor(mat_v3(m.base_color), mat_v3(m.specular_color), wh) * (m.specular_weight * micro), pdfH);
            if (wGlass > 0.f && rough) { const float F = fresnel_exact(wh, eta); add(1, wGlass, f3(F * micro, F * micro, F * micro), F * pdfH); }
            if (wGloss > 0.f) {
                float3 f = mat_v3(m.base_color) * (glossKd * CWPB_INV_PI * terminator_shadowing(nr, wi));
                float pdf = (1.f - glossPSpec) * wi.z * CWPB_INV_PI;
                if (rough && glossF > 0.f) {
                    const float s = m.specular_weight * fresnel_exact(wh, m.ior) * micro;
                    f = f + f3(s, s, s); pdf += glossPSpec * pdfH;
                }
                add(2, wGloss, f, pdf);
            }
        } else if (wi.z < 0.f && wGlass > 0.f && !ggx.smooth) {
            // refraction through the glass base: generalised half vector h ~ wo + eta wi on the wo side
            float3 h = normalize(wo + wi * eta);
            if (h.z < 0.f) h = -h;
            const float wh = dot(wo, h), ih = dot(wi, h);
            const float F = wh > 0.f && ih < 0.f ? fresnel_exact(wh, eta) : 1.f;
            if (F < 1.f) {
                const float den = wh + eta * ih;
                const float jacobian = eta * eta * -ih / (den * den);   // |dh / dwi|
                add(1, wGlass, mat_v3(m.base_color) * ((1.f - F) * ggx.D(h.z) * ggx.G2(wo.z, -wi.z) * wh * jacobian / (wo.z * -wi.z)),
                    (1.f - F) * ggx.visible_pdf(wo, h) * jacobian);
            }
        }
        if (ownPdf) *ownPdf = o;
        return r;
    }

    // a direction from one base, chosen by u; the weight covers the whole material
    CWPB_HD bool sample(float3 wo, float u, float u1, float u2, float3& wi, float3& w, float& pdf) const {
        int base; float uu = 0.f;
        if (u < wMetal) base = 0;
        else if (u < wMetal + wGlass) { base = 1; uu = fminf((u - wMetal) / wGlass, 0.99999994f); }
        else { base = 2; uu = fminf(wGloss > 0.f ? (u - wMetal - wGlass) / wGloss : 0.f, 0.99999994f); }
        bool delta = false;
        if (base == 0) {
            if (ggx.smooth) {
                wi = f3(-wo.x, -wo.y, wo.z);
                w = fresnel_conductor(mat_v3(m.base_color), mat_v3(m.specular_color), wo.z) * m.specular_weight;
                delta = true;
            } else {
                const float3 h = ggx.sample_visible(wo, u1, u2);
                const float wh = dot(wo, h);
                wi = reflect_about(wo, h, wh);
                if (wi.z <= 0.f || wh <= 0.f) return false;
                // f cos / pdf of the conductor alone: F ws G2 / G1(wo)
                w = fresnel_conductor(mat_v3(m.base_color), mat_v3(m.specular_color), wh) * (m.specular_weight * ggx.G2(wo.z, wi.z) / ggx.G1(wo.z));
                pdf = ggx.visible_pdf(wo, h) / (4.f * wh);
            }
        } else if (base == 1) {
            const float3 h = ggx.smooth ? f3(0.f, 0.f, 1.f) : ggx.sample_visible(wo, u1, u2);
            const float wh = dot(wo, h);
            if (wh <= 0.f) return false;
            if (uu < fresnel_exact(wh, eta)) {   // reflect
                wi = reflect_about(wo, h, wh);
                if (wi.z <= 0.f) return false;
                if (ggx.smooth) { w = f3(1.f, 1.f, 1.f); delta = true; }
            } else {                              // refract (Snell's law about h)
                const float cosT = sqrtf(fmaxf(1.f - (1.f - wh * wh) / (eta * eta), 0.f));
                wi = wo * (-1.f / eta) + h * (wh / eta - cosT);
                if (wi.z >= 0.f) return false;
                wi = normalize(wi);
                if (ggx.smooth) { w = mat_v3(m.base_color); delta = true; }
            }
        } else {
            if (uu < glossPSpec) {
                if (ggx.smooth) { wi = f3(-wo.x, -wo.y, wo.z); const float s = glossF / glossPSpec; w = f3(s, s, s); delta = true; }
                else {
                    const float3 h = ggx.sample_visible(wo, u1, u2);
                    wi = reflect_about(wo, h, dot(wo, h));
                    if (wi.z <= 0.f) return false;
                }
            } else {
                wi = cosine_dir(f3(0.f, 0.f, 1.f), u1, u2);
                if (wi.z <= 0.f) return false;
            }
        }
        if (delta) { pdf = 0.f; return true; }                       // no other base has density on a Dirac lobe
        if (base == 0 && wMetal == 1.f) return true;                  // the metal alone: its closed-form weight
        float ownPdf;
        const BsdfValue e = eval(wo, wi, base, &ownPdf);
        if (base != 0 && !(ownPdf > 0.f)) return false;               // the sampled base has no density there
        // (with one base of weight 1 the material's f and pdf are that base's own, so one formula covers both)
        if (e.pdf <= 0.f) return false;
        w = e.f * (fabsf(wi.z) / e.pdf); pdf = e.pdf;
        return true;
    }
};

// some lobe of the material has a density, so light sampling can contribute
CWPB_HD bool has_non_delta(const cwp_material& m) {
    const float wMetal = m.metallic, wGlass = (1.f - m.metallic) * m.transmission, wGloss = (1.f - m.metallic) * (1.f - m.transmission);
    const bool rough = m.roughness * m.roughness >= kSmoothAlpha;
    return (wGloss > 0.f && (rough || luminance(mat_v3(m.base_color)) > 0.f)) || (rough && (wMetal > 0.f || wGlass > 0.f));
}
// f and pdf of the material; nr is the unperturbed normal for the terminator term (+z: off)
CWPB_HD BsdfValue bsdf_eval(const cwp_material& m, float3 wo, float3 wi, float etaRel, int gdEnergy, float ux1, float ux2, float3 nr = f3(0.f, 0.f, 1.f)) {
    return PbrVertex(m, wo, etaRel, gdEnergy, ux1, ux2, nr).eval(wo, wi);
}
CWPB_HD bool bsdf_sample(const cwp_material& m, float3 wo, float etaRel, int gdEnergy, float ux1, float ux2, float u, float u1, float u2,
                         float3& wi, float3& weight, float& pdf, float3 nr = f3(0.f, 0.f, 1.f)) {
    return PbrVertex(m, wo, etaRel, gdEnergy, ux1, ux2, nr).sample(wo, u, u1, u2, wi, weight, pdf);
}
// power heuristic with exponent 2
CWPB_HD float mis_power(float a, float b) { const float a2 = a * a; return a2 / (a2 + b * b); }

}  // namespace cwpb
