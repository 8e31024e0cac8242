// host_lights.cpp - light tables of the emissive triangles of an instanced scene at one frame.
//
// Follows SceneSetup::frameData (app/scene_setup.cpp:274-299): instances in order, each one's emissive triangles in
// mesh order, corners transformed in float by the 3x4 rows, area = 0.5 |e1 x e2| in float, power = luminance x area
// accumulated in double, CDF entries rounded from the double prefix sums, the last one set to 1; the area density of
// a material is luminance(emission) / total power. The reference's triangle reference in the first record is its BVH
// leaf position (its uv table is in leaf order); here it is the global triangle id, which addresses the uv table of the
// serving form (mesh order).
#include "lights.h"
#include "runtime.h"
#include <cmath>
#include <cstring>

namespace cwpb {

static float lum(const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }   // render/bsdf.h:19

void emissive_set(const float* soup, const int* meshFirst, int nMesh, const int* meshMat, const cwp_material* mats, int nMats, EmissiveSet& out) {
    out.first.assign((size_t)nMesh + 1, 0); out.tris.clear();
    bool any = false;
    for (int j = 0; j < nMats; j++) any = any || is_emissive(mats[j]);
    for (int m = 0; m < nMesh; m++) {
        out.first[m] = (int)out.tris.size();
        if (!any) continue;
        for (int g = meshFirst[m]; g < meshFirst[m + 1]; g++) {
            const float* r = soup + 12 * (size_t)g;
            int fm; memcpy(&fm, r + 7, 4);
            int mid = meshMat[m] + fm; mid = mid < 0 ? 0 : mid >= nMats ? nMats - 1 : mid;
            if (!is_emissive(mats[mid])) continue;
            EmissiveTri e; e.mat = mid; e.gtri = g;
            for (int k = 0; k < 3; k++) for (int c = 0; c < 3; c++) e.v[3 * k + c] = r[4 * k + c];
            out.tris.push_back(e);
        }
    }
    out.first[nMesh] = (int)out.tris.size();
}

void frame_lights(const EmissiveSet& S, const float* xf, const int* instMesh, int64_t nInst, const cwp_material* mats, int nMats,
                  std::vector<float>& emT, std::vector<float>& emC, std::vector<float>& mlp) {
    emT.clear(); emC.clear(); mlp.assign((size_t)nMats, 0.f);
    if (S.empty()) return;
    std::vector<double> pw; double tot = 0;
    for (int64_t i = 0; i < nInst; i++) {
        const float* m = xf + 12 * i; const int mesh = instMesh[i];
        for (int k = S.first[mesh]; k < S.first[mesh + 1]; k++) {
            const EmissiveTri& E = S.tris[k];
            float w[3][3];
            for (int c = 0; c < 3; c++) {
                const float* p = E.v + 3 * c;
                for (int r = 0; r < 3; r++) w[c][r] = m[4 * r] * p[0] + m[4 * r + 1] * p[1] + m[4 * r + 2] * p[2] + m[4 * r + 3];
            }
            const float e1[3] = { w[1][0] - w[0][0], w[1][1] - w[0][1], w[1][2] - w[0][2] };
            const float e2[3] = { w[2][0] - w[0][0], w[2][1] - w[0][1], w[2][2] - w[0][2] };
            const float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
            const double area = 0.5 * sqrtf(cx * cx + cy * cy + cz * cz);
            float idf, mf; memcpy(&idf, &E.gtri, 4); memcpy(&mf, &E.mat, 4);
            const float rec[12] = { w[0][0], w[0][1], w[0][2], idf, e1[0], e1[1], e1[2], mf, e2[0], e2[1], e2[2], 0.f };
            emT.insert(emT.end(), rec, rec + 12);
            double pwr = lum(mats[E.mat].emission) * area; pwr = pwr > 0 ? pwr : 0;
            pw.push_back(pwr); tot += pwr;
        }
    }
    if (!(tot > 0)) { emT.clear(); return; }
    emC.assign(pw.size() + 1, 0.f);
    double c = 0;
    for (size_t e = 0; e < pw.size(); e++) { c += pw[e]; emC[e + 1] = (float)(c / tot); }
    emC.back() = 1.f;
    for (int j = 0; j < nMats; j++) if (is_emissive(mats[j])) mlp[j] = (float)(lum(mats[j].emission) / tot);
}

}  // namespace cwpb

using namespace cwpb;

extern "C" int cwp_emissive_tables(const cwp_mesh_view* meshes, int32_t nMeshes, const int32_t* meshMatBase, const cwp_material* mats, int32_t nMats,
                                   const float* xforms, const int32_t* instMesh, int64_t nInst, float* emTris, float* emCdf, float* matPdf, int64_t* nEm) {
    CWPB_CHECK(meshes && nMeshes >= 1 && meshMatBase && mats && nMats >= 1 && nEm && nInst >= 0 && (nInst == 0 || (xforms && instMesh)), CWP_ERR_INVALID,
               "NULL argument");
    std::vector<int> first((size_t)nMeshes + 1, 0);
    for (int m = 0; m < nMeshes; m++) {
        const cwp_mesh_view& v = meshes[m];
        CWPB_CHECK(v.verts && v.faces && v.n_tris > 0 && v.n_verts > 0, CWP_ERR_INVALID, "mesh %d is empty or has NULL arrays", m);
        CWPB_CHECK((int64_t)first[m] + v.n_tris < (1ll << 30), CWP_ERR_INVALID, "more than 2^30 triangles");
        first[m + 1] = first[m] + (int)v.n_tris;
    }
    for (int64_t i = 0; i < nInst; i++) CWPB_CHECK(instMesh[i] >= 0 && instMesh[i] < nMeshes, CWP_ERR_INVALID, "instance %lld: mesh %d out of range", (long long)i, instMesh[i]);
    std::vector<float> soup((size_t)12 * first[nMeshes], 0.f);
    for (int m = 0; m < nMeshes; m++) {
        const cwp_mesh_view& v = meshes[m];
        for (int64_t t = 0; t < v.n_tris; t++) {
            float* r = &soup[(size_t)12 * (first[m] + t)];
            for (int k = 0; k < 3; k++) {
                const int vi = v.faces[3 * t + k];
                CWPB_CHECK(vi >= 0 && vi < v.n_verts, CWP_ERR_INVALID, "mesh %d triangle %lld: vertex index %d out of range", m, (long long)t, vi);
                memcpy(r + 4 * k, v.verts + 3 * (size_t)vi, 12);
            }
            const int id = (int)t, fm = v.face_mat ? v.face_mat[t] : 0;
            memcpy(r + 3, &id, 4); memcpy(r + 7, &fm, 4);
        }
    }
    EmissiveSet S;
    emissive_set(soup.data(), first.data(), nMeshes, meshMatBase, mats, nMats, S);
    std::vector<float> emT, emC, mlp;
    frame_lights(S, xforms, instMesh, nInst, mats, nMats, emT, emC, mlp);
    *nEm = (int64_t)emT.size() / 12;
    if (!emTris) return CWP_OK;
    CWPB_CHECK(emCdf && matPdf, CWP_ERR_INVALID, "NULL output");
    memcpy(emTris, emT.data(), emT.size() * sizeof(float));
    memcpy(emCdf, emC.data(), emC.size() * sizeof(float));
    memcpy(matPdf, mlp.data(), mlp.size() * sizeof(float));
    return CWP_OK;
}
