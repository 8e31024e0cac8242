// bsdf.cuh - OpenPBR-subset materials (host + device) for the serving form's integrator.
//
// cwp_material (64 B) blends three bases linearly: metallic -> rough conductor; (1 - metallic) transmission -> rough
// dielectric (reflection + refraction); the rest -> glossy-diffuse (a GGX dielectric specular lobe over a Lambertian
// base). Roughness r gives GGX alpha = r^2; alpha below kDeltaAlpha is a perfectly specular lobe. The semantics follow
// the reference's render/bsdf.h and scene/material.h (same lobes, weights and sample weights, so images agree); the
// formulas are those of the cited papers:
//   GGX distribution, height-correlated Smith masking-shadowing ... Walter et al. 2007; Heitz, JCGT 2014
//   visible-normal sampling with spherical caps .................. Dupuy & Benyoub, HPG 2023
//   exact unpolarised dielectric Fresnel, rough refraction ....... Walter et al. 2007 (energy convention: no eta^2)
//   conductor Fresnel: Schlick with the F82 tint term ............ Kutz et al. 2021, as specified by OpenPBR 1.0
// Frame: z = shading normal, wo.z > 0 (towards the viewer). eval() returns f and the solid-angle pdf of the non-delta
// lobes; sample() returns wi, weight = f |cos| / pdf and pdf (0 marks a delta sample).
#pragma once
#include "cwp_b200.h"
#include "vecmath.h"

namespace cwpb {

static constexpr float kDeltaAlpha = 1e-3f;
#define CWPB_PI 3.14159265f

CWPB_HD float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
CWPB_HD float3 mat_v3(const float* a) { return f3(a[0], a[1], a[2]); }

// ---- microfacet terms ----
CWPB_HD float ggx_ndf(float cosM, float a2) {
    if (cosM <= 0.f) return 0.f;
    const float c2 = cosM * cosM, k = c2 * (a2 - 1.f) + 1.f;
    return a2 / (CWPB_PI * k * k);
}
CWPB_HD float smith_lambda(float cosW, float a2) {
    const float c2 = cosW * cosW;
    if (c2 < 1e-12f) return 1e12f;
    return 0.5f * (sqrtf(1.f + a2 * (1.f - c2) / c2) - 1.f);
}
CWPB_HD float smith_g1(float cosW, float a2) { return 1.f / (1.f + smith_lambda(cosW, a2)); }
CWPB_HD float smith_g2(float cosO, float cosI, float a2) { return 1.f / (1.f + smith_lambda(cosO, a2) + smith_lambda(cosI, a2)); }
// density of the normals visible from wo: G1(wo) max(0, wo.m) D(m) / wo.z
CWPB_HD float vndf_pdf(float3 wo, float3 m, float a2) {
    const float om = dot(wo, m);
    if (om <= 0.f || m.z <= 0.f) return 0.f;
    return smith_g1(wo.z, a2) * om * ggx_ndf(m.z, a2) / wo.z;
}
// a visible normal: the hemisphere configuration of wo stretched to alpha 1, a uniform point on the spherical cap
// below it, shifted by the stretched view direction and unstretched
CWPB_HD float3 vndf_sample(float3 wo, float a, float u1, float u2) {
    const float3 v = normalize(f3(a * wo.x, a * wo.y, wo.z));
    const float phi = CWPB_TWO_PI * u1;
    const float z = (1.f - u2) * (1.f + v.z) - v.z;
    const float s = sqrtf(fminf(fmaxf(1.f - z * z, 0.f), 1.f));
    const float3 h = f3(s * cosf(phi) + v.x, s * sinf(phi) + v.y, z + v.z);
    return normalize(f3(a * h.x, a * h.y, fmaxf(h.z, 0.f)));
}

// ---- Fresnel ----
// unpolarised dielectric reflectance; cosI > 0 on the incident side, eta = n_transmitted / n_incident
CWPB_HD float fresnel_dielectric(float cosI, float eta) {
    const float sin2T = (1.f - cosI * cosI) / (eta * eta);
    if (sin2T >= 1.f) return 1.f;   // total internal reflection
    const float cosT = sqrtf(1.f - sin2T);
    const float rs = (cosI - eta * cosT) / (cosI + eta * cosT), rp = (eta * cosI - cosT) / (eta * cosI + cosT);
    return 0.5f * (rs * rs + rp * rp);
}
// Schlick's curve from F0 minus b mu (1 - mu)^6, with b chosen so that the curve equals tint x Schlick at
// mu = 1/7 (the angle of the F82 measurement): F82 tint correction of OpenPBR's conductor
CWPB_HD float3 fresnel_f82(float3 F0, float3 tint, float mu) {
    mu = fminf(fmaxf(mu, 0.f), 1.f);
    const float q = 1.f - mu, q2 = q * q, q5 = q2 * q2 * q, q6 = q5 * q;
    const float mb = 1.f / 7.f, qb = 6.f / 7.f, qb2 = qb * qb, qb5 = qb2 * qb2 * qb, qb6 = qb5 * qb;
    const float3 one = f3(1.f, 1.f, 1.f);
    const float3 schlick = F0 + (one - F0) * q5;
    const float3 schlickB = F0 + (one - F0) * qb5;
    const float3 b = schlickB * (one - tint) * (1.f / (mb * qb6));
    const float3 F = schlick - b * (mu * q6);
    return f3(fminf(fmaxf(F.x, 0.f), 1.f), fminf(fmaxf(F.y, 0.f), 1.f), fminf(fmaxf(F.z, 0.f), 1.f));
}

struct BsdfValue { float3 f; float pdf; };

// ---- glossy-diffuse base: GGX dielectric specular (weight ws, ior) + Lambertian base colour weighted by kd ----
// energy = 0: kd = 1 - ws F(wo.z). energy = 1: kd = 1 - X with X = ws F(wo.m) G2 / G1(wo) for one visible normal m
// drawn from (ux1, ux2), an unbiased estimate of the specular lobe's directional albedo. Lobe choice uses F(wo.z).
// bump-terminator shadowing of the diffuse lobe (Chiang, Li, Burley, "Taming the Shadow Terminator", SIGGRAPH 2019
// talk): nr = the unperturbed normal in the frame of the mapped shading normal, g = (nr . wi) / (wi.z nr.z), G = g +
// g^2 - g^3 on [0, 1), 1 above, 0 below; nr = +z gives G = 1 exactly (the term off)
CWPB_HD float bump_shadowing(float3 nr, float3 wi) {
    if (nr.z >= 1.f) return 1.f;
    const float g = dot(nr, wi) / (wi.z * nr.z);
    if (g >= 1.f) return 1.f;
    if (g < 0.f) return 0.f;
    return g + g * g - g * g * g;
}

struct GlossyDiffuseLobe {
    float3 base; float ws, eta, a, a2, Fo, pSpec, kd; bool delta; float3 nr = f3(0.f, 0.f, 1.f);
    CWPB_HD GlossyDiffuseLobe(const cwp_material& m, float3 wo, int energy, float ux1, float ux2) {
        base = mat_v3(m.base_color); ws = m.specular_weight; eta = m.ior; a = m.roughness * m.roughness; a2 = a * a; delta = a < kDeltaAlpha;
        Fo = ws > 0.f ? ws * fresnel_dielectric(wo.z, eta) : 0.f;
        const float pd = (1.f - Fo) * luminance(base);
        pSpec = Fo + pd > 0.f ? Fo / (Fo + pd) : 0.f;
        kd = 1.f - Fo;
        if (energy && ws > 0.f && !delta) {
            const float3 mm = vndf_sample(wo, a, ux1, ux2);
            const float om = dot(wo, mm);
            const float3 wr = mm * (2.f * om) - wo;
            const float X = (om > 0.f && wr.z > 0.f) ? ws * fresnel_dielectric(om, eta) * smith_g2(wo.z, wr.z, a2) / smith_g1(wo.z, a2) : 0.f;
            kd = 1.f - X;
        }
        kd = fmaxf(kd, 0.f);
    }
    CWPB_HD BsdfValue eval(float3 wo, float3 wi) const {
        BsdfValue r{ f3(0.f, 0.f, 0.f), 0.f };
        if (wi.z <= 0.f) return r;
        r.f = base * (kd * CWPB_INV_PI * bump_shadowing(nr, wi)); r.pdf = (1.f - pSpec) * wi.z * CWPB_INV_PI;
        if (!delta && Fo > 0.f) {
            const float3 m = normalize(wo + wi); const float om = dot(wo, m);
            if (om > 0.f) {
                const float spec = ws * fresnel_dielectric(om, eta) * ggx_ndf(m.z, a2) * smith_g2(wo.z, wi.z, a2) / (4.f * wo.z * wi.z);
                r.f = r.f + f3(spec, spec, spec); r.pdf += pSpec * vndf_pdf(wo, m, a2) / (4.f * om);
            }
        }
        return r;
    }
    CWPB_HD bool sample(float3 wo, float u, float u1, float u2, float3& wi, float3& w, float& pdf) const {
        if (u < pSpec) {
            if (delta) { wi = f3(-wo.x, -wo.y, wo.z); const float s = Fo / pSpec; w = f3(s, s, s); pdf = 0.f; return true; }
            const float3 m = vndf_sample(wo, a, u1, u2); wi = m * (2.f * dot(wo, m)) - wo;
            if (wi.z <= 0.f) return false;
        } else {
            wi = cosine_dir(f3(0.f, 0.f, 1.f), u1, u2);
            if (wi.z <= 0.f) return false;
        }
        const BsdfValue e = eval(wo, wi);
        if (e.pdf <= 0.f) return false;
        w = e.f * (wi.z / e.pdf); pdf = e.pdf; return true;
    }
};

// ---- metallic base: rough conductor, F = ws F82(base colour, specular colour) ----
struct ConductorLobe {
    float3 F0, tint; float ws, a, a2; bool delta;
    CWPB_HD explicit ConductorLobe(const cwp_material& m) { F0 = mat_v3(m.base_color); tint = mat_v3(m.specular_color); ws = m.specular_weight; a = m.roughness * m.roughness; a2 = a * a; delta = a < kDeltaAlpha; }
    CWPB_HD BsdfValue eval(float3 wo, float3 wi) const {
        BsdfValue r{ f3(0.f, 0.f, 0.f), 0.f };
        if (delta || wi.z <= 0.f) return r;
        const float3 m = normalize(wo + wi); const float om = dot(wo, m);
        if (om <= 0.f) return r;
        r.f = fresnel_f82(F0, tint, om) * (ws * ggx_ndf(m.z, a2) * smith_g2(wo.z, wi.z, a2) / (4.f * wo.z * wi.z));
        r.pdf = vndf_pdf(wo, m, a2) / (4.f * om);
        return r;
    }
    CWPB_HD bool sample(float3 wo, float u1, float u2, float3& wi, float3& w, float& pdf) const {
        if (delta) { wi = f3(-wo.x, -wo.y, wo.z); w = fresnel_f82(F0, tint, wo.z) * ws; pdf = 0.f; return true; }
        const float3 m = vndf_sample(wo, a, u1, u2); const float om = dot(wo, m);
        wi = m * (2.f * om) - wo;
        if (wi.z <= 0.f || om <= 0.f) return false;
        w = fresnel_f82(F0, tint, om) * (ws * smith_g2(wo.z, wi.z, a2) / smith_g1(wo.z, a2));   // F G2 / G1(wo)
        pdf = vndf_pdf(wo, m, a2) / (4.f * om);
        return true;
    }
};

// ---- transmissive base: rough dielectric; eta = n(other side) / n(wo side); refraction tinted by the base colour ----
struct DielectricLobe {
    float3 tint; float eta, a, a2; bool delta;
    CWPB_HD DielectricLobe(const cwp_material& m, float etaRel) { tint = mat_v3(m.base_color); eta = etaRel; a = m.roughness * m.roughness; a2 = a * a; delta = a < kDeltaAlpha; }
    CWPB_HD BsdfValue eval(float3 wo, float3 wi) const {
        BsdfValue r{ f3(0.f, 0.f, 0.f), 0.f };
        if (delta) return r;
        if (wi.z > 0.f) {
            const float3 m = normalize(wo + wi); const float om = dot(wo, m);
            if (om <= 0.f) return r;
            const float F = fresnel_dielectric(om, eta);
            const float s = F * ggx_ndf(m.z, a2) * smith_g2(wo.z, wi.z, a2) / (4.f * wo.z * wi.z);
            r.f = f3(s, s, s); r.pdf = F * vndf_pdf(wo, m, a2) / (4.f * om);
        } else if (wi.z < 0.f) {
            float3 m = normalize(wo + wi * eta);   // generalised half vector of refraction
            if (m.z < 0.f) m = -m;
            const float om = dot(wo, m), im = dot(wi, m);
            if (om <= 0.f || im >= 0.f) return r;
            const float F = fresnel_dielectric(om, eta);
            if (F >= 1.f) return r;
            const float den = om + eta * im, jac = eta * eta * (-im) / (den * den);   // |dm / dwi|
            const float s = (1.f - F) * ggx_ndf(m.z, a2) * smith_g2(wo.z, -wi.z, a2) * om * jac / (wo.z * -wi.z);
            r.f = tint * s; r.pdf = (1.f - F) * vndf_pdf(wo, m, a2) * jac;
        }
        return r;
    }
    CWPB_HD bool sample(float3 wo, float u, float u1, float u2, float3& wi, float3& w, float& pdf) const {
        const float3 m = delta ? f3(0.f, 0.f, 1.f) : vndf_sample(wo, a, u1, u2);
        const float om = dot(wo, m);
        if (om <= 0.f) return false;
        const float F = fresnel_dielectric(om, eta);
        if (u < F) {
            wi = m * (2.f * om) - wo;
            if (wi.z <= 0.f) return false;
            if (delta) { w = f3(1.f, 1.f, 1.f); pdf = 0.f; return true; }
        } else {
            const float cosT = sqrtf(fmaxf(1.f - (1.f - om * om) / (eta * eta), 0.f));
            wi = wo * (-1.f / eta) + m * (om / eta - cosT);
            if (wi.z >= 0.f) return false;
            wi = normalize(wi);
            if (delta) { w = tint; pdf = 0.f; return true; }
        }
        const BsdfValue e = eval(wo, wi);
        if (e.pdf <= 0.f) return false;
        w = e.f * (fabsf(wi.z) / e.pdf); pdf = e.pdf; return true;
    }
};

// ---- the blended material ----
CWPB_HD void base_weights(const cwp_material& m, float& wM, float& wT, float& wD) {
    wM = m.metallic; wT = (1.f - m.metallic) * m.transmission; wD = (1.f - m.metallic) * (1.f - m.transmission);
}
// some lobe has a density (light sampling can help)
CWPB_HD bool has_non_delta(const cwp_material& m) {
    float wM, wT, wD; base_weights(m, wM, wT, wD);
    const bool rough = m.roughness * m.roughness >= kDeltaAlpha;
    return (wD > 0.f && (luminance(mat_v3(m.base_color)) > 0.f || rough)) || ((wM > 0.f || wT > 0.f) && rough);
}
// nr: the unperturbed normal for the bump-terminator term, +z = off
CWPB_HD BsdfValue bsdf_eval(const cwp_material& m, float3 wo, float3 wi, float etaRel, int gdEnergy, float ux1, float ux2, float3 nr = f3(0.f, 0.f, 1.f)) {
    float wM, wT, wD; base_weights(m, wM, wT, wD);
    BsdfValue r{ f3(0.f, 0.f, 0.f), 0.f };
    if (wM > 0.f) { const BsdfValue e = ConductorLobe(m).eval(wo, wi); r.f = r.f + e.f * wM; r.pdf += wM * e.pdf; }
    if (wT > 0.f) { const BsdfValue e = DielectricLobe(m, etaRel).eval(wo, wi); r.f = r.f + e.f * wT; r.pdf += wT * e.pdf; }
    if (wD > 0.f) { GlossyDiffuseLobe g(m, wo, gdEnergy, ux1, ux2); g.nr = nr; const BsdfValue e = g.eval(wo, wi); r.f = r.f + e.f * wD; r.pdf += wD * e.pdf; }
    return r;
}
// one base chosen by u (one-sample MIS over the bases); weight of the whole material, pdf 0 for delta samples
CWPB_HD bool bsdf_sample(const cwp_material& m, float3 wo, float etaRel, int gdEnergy, float ux1, float ux2, float u, float u1, float u2,
                         float3& wi, float3& weight, float& pdf, float3 nr = f3(0.f, 0.f, 1.f)) {
    float wM, wT, wD; base_weights(m, wM, wT, wD);
    bool ok;
    if (u < wM) ok = ConductorLobe(m).sample(wo, u1, u2, wi, weight, pdf);
    else if (u < wM + wT) ok = DielectricLobe(m, etaRel).sample(wo, fminf((u - wM) / wT, 0.99999994f), u1, u2, wi, weight, pdf);
    else { GlossyDiffuseLobe g(m, wo, gdEnergy, ux1, ux2); g.nr = nr; ok = g.sample(wo, fminf(wD > 0.f ? (u - wM - wT) / wD : 0.f, 0.99999994f), u1, u2, wi, weight, pdf); }
    if (!ok) return false;
    if (pdf <= 0.f) return true;                          // a delta sample: no other base has density there
    if (wM == 1.f || wT == 1.f || wD == 1.f) return true;  // one base: its own weight is already f |cos| / pdf
    const BsdfValue e = bsdf_eval(m, wo, wi, etaRel, gdEnergy, ux1, ux2, nr);
    if (e.pdf <= 0.f) return false;
    weight = e.f * (fabsf(wi.z) / e.pdf); pdf = e.pdf;
    return true;
}
// power heuristic (Veach 1997), beta = 2
CWPB_HD float mis_power(float a, float b) { const float a2 = a * a; return a2 / (a2 + b * b); }

}  // namespace cwpb
