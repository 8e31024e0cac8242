// host_env.cpp - environment maps for the serving integrator: a Radiance RGBE (.hdr) reader and the importance-
// sampling tables of an equirectangular map (texel radiance, marginal CDF over rows, conditional CDF per row, texel
// weight = luminance x sin(theta)).
//
// The tables follow the reference's buildEnvMap (scene/environment.cpp:7-38) operation for operation, in double as
// it does, so a map gives the same float tables bit for bit; the RGBE decoding (mantissa x 2^(exponent - 136), no
// half-step offset) follows its loadHDR (io/hdr_image.cpp:7-11) so a file gives the same radiance.
#include "cwp_b200.h"
#include "runtime.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

void rgbe_to_rgb(const unsigned char* e, float* out) {
    if (e[3] == 0) { out[0] = out[1] = out[2] = 0.f; return; }
    const float f = ldexpf(1.f, (int)e[3] - 136);
    out[0] = e[0] * f; out[1] = e[1] * f; out[2] = e[2] * f;
}

struct File {
    FILE* f = nullptr;
    explicit File(const char* p) : f(fopen(p, "rb")) {}
    ~File() { if (f) fclose(f); }
};

// one scanline of w RGBE pixels: the run-length form (four channels one after the other) or a flat line
int read_scanline(FILE* fp, int w, unsigned char* scan, const char* path) {
    unsigned char hd[4];
    CWPB_CHECK(fread(hd, 1, 4, fp) == 4, CWP_ERR_IO, "%s: truncated", path);
    if (w >= 8 && w < 32768 && hd[0] == 2 && hd[1] == 2 && ((hd[2] << 8) | hd[3]) == w) {
        for (int c = 0; c < 4; c++) {
            for (int x = 0; x < w;) {
                int n = fgetc(fp);
                CWPB_CHECK(n != EOF && n != 0, CWP_ERR_IO, "%s: truncated or corrupt run", path);
                if (n > 128) {
                    n -= 128;
                    const int v = fgetc(fp);
                    CWPB_CHECK(v != EOF && x + n <= w, CWP_ERR_IO, "%s: corrupt run", path);
                    for (int k = 0; k < n; k++) scan[4 * (x++) + c] = (unsigned char)v;
                } else {
                    CWPB_CHECK(x + n <= w, CWP_ERR_IO, "%s: corrupt run", path);
                    for (int k = 0; k < n; k++) {
                        const int v = fgetc(fp);
                        CWPB_CHECK(v != EOF, CWP_ERR_IO, "%s: truncated", path);
                        scan[4 * (x++) + c] = (unsigned char)v;
                    }
                }
            }
        }
    } else {
        memcpy(scan, hd, 4);
        CWPB_CHECK(w == 1 || fread(scan + 4, 1, (size_t)(w - 1) * 4, fp) == (size_t)(w - 1) * 4, CWP_ERR_IO, "%s: truncated", path);
    }
    return CWP_OK;
}

}  // namespace

extern "C" int cwp_hdr_load(const char* path, int32_t* w, int32_t* h, float* rgb) {
    CWPB_CHECK(path && w && h, CWP_ERR_INVALID, "NULL argument");
    File F(path);
    CWPB_CHECK(F.f, CWP_ERR_IO, "cannot open %s", path);
    char line[512];
    CWPB_CHECK(fgets(line, sizeof line, F.f) && (strncmp(line, "#?RADIANCE", 10) == 0 || strncmp(line, "#?RGBE", 6) == 0), CWP_ERR_IO,
               "%s is not a Radiance file", path);
    bool fmtOk = true;
    while (fgets(line, sizeof line, F.f)) {
        if (line[0] == '\n' || line[0] == '\r') break;
        if (strncmp(line, "FORMAT=", 7) == 0 && strncmp(line + 7, "32-bit_rle_rgbe", 15) != 0) fmtOk = false;
    }
    CWPB_CHECK(fmtOk, CWP_ERR_IO, "%s: only FORMAT=32-bit_rle_rgbe is read", path);
    int hh = 0, ww = 0;
    CWPB_CHECK(fgets(line, sizeof line, F.f) && sscanf(line, "-Y %d +X %d", &hh, &ww) == 2 && ww > 0 && hh > 0 && (int64_t)ww * hh < (1ll << 28),
               CWP_ERR_IO, "%s: only the '-Y H +X W' orientation is read", path);
    *w = ww; *h = hh;
    if (!rgb) return CWP_OK;   // size query
    std::vector<unsigned char> scan((size_t)ww * 4);
    for (int y = 0; y < hh; y++) {
        if (int rc = read_scanline(F.f, ww, scan.data(), path)) return rc;
        for (int x = 0; x < ww; x++) rgbe_to_rgb(&scan[4 * x], rgb + ((size_t)y * ww + x) * 3);
    }
    return CWP_OK;
}

extern "C" int cwp_envmap_build(const float* rgb, int32_t w, int32_t h, float strength, float* texels, float* marg, float* cond) {
    CWPB_CHECK(rgb && texels && marg && cond, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(w > 0 && h > 0 && (int64_t)w * h < (1ll << 28), CWP_ERR_INVALID, "environment map %dx%d", w, h);
    CWPB_CHECK(std::isfinite(strength) && strength >= 0.f, CWP_ERR_INVALID, "environment strength %g", strength);
    const double pi = 3.14159265358979323846;
    std::vector<double> rowSum(h, 0.0), rowCdf((size_t)w + 1);
    for (int y = 0; y < h; y++) {
        const double st = sin(pi * (y + 0.5) / h);   // solid angle of the row's texels is proportional to sin(theta)
        rowCdf[0] = 0.0;
        for (int x = 0; x < w; x++) {
            const float* c = rgb + ((size_t)y * w + x) * 3;
            const float r = c[0] * strength, g = c[1] * strength, b = c[2] * strength;
            float* t = texels + 4 * ((size_t)y * w + x);
            t[0] = r; t[1] = g; t[2] = b; t[3] = 0.f;
            const double lum = 0.2126 * r + 0.7152 * g + 0.0722 * b;
            rowCdf[x + 1] = rowCdf[x] + (lum > 0 ? lum : 0.0) * st;
        }
        rowSum[y] = rowCdf[w];
        float* cr = cond + (size_t)y * (w + 1);
        for (int x = 0; x <= w; x++) cr[x] = rowSum[y] > 0 ? (float)(rowCdf[x] / rowSum[y]) : (float)x / w;
        cr[w] = 1.f;
    }
    std::vector<double> mc((size_t)h + 1, 0.0);
    for (int y = 0; y < h; y++) mc[y + 1] = mc[y] + rowSum[y];
    const double tot = mc[h];
    for (int y = 0; y <= h; y++) marg[y] = tot > 0 ? (float)(mc[y] / tot) : (float)y / h;
    marg[h] = 1.f;
    return CWP_OK;
}
