// Host-side pieces around the solver that a headless driver needs: OBJ
// ingestion, model placement, the triangle buffer LBM_SetSolidMesh takes,
// the Reynolds-number-to-tau rule and the Strouhal post-processing.
//
// Reference behaviour restated here:
//   simulation/obj-file-loader/lib/model_loader.c:8-151  (loadOBJ)
//   simulation/src/model_bounds.c:146-287                (bounds, triangles)
//   simulation/src/main.c:251-349                        (auto scale/orient/shift)
//   simulation/src/main.c:438-460                        (Re -> tau, clamp)
//   simulation/src/drag_metrics.c:8-68                   (Strouhal)
// Arithmetic keeps the reference's types (float, with the double
// intermediate of `rotationY * M_PI / 180.0f` in model_bounds.c), so the
// triangles are bit-identical to the reference's on the same file.
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/lattice_lbm.h"

namespace {

int count_lines_with(const char *path, char c0) {
    // model_loader.c:8-44 (256-byte line buffer, "v " / "f " prefixes)
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    int n = 0;
    char line[256];
    while (fgets(line, sizeof(line), f))
        if (line[0] == c0 && line[1] == ' ') n++;
    fclose(f);
    return n;
}

int parse_index(const char *token) {
    // model_loader.c:48-52: the leading integer of "v", "v/vt", "v/vt/vn", "v//vn"
    int v = 0;
    sscanf(token, "%d", &v);
    return v;
}

void read_token(char *&p, char *out) {
    int i = 0;
    while (*p && *p != ' ' && *p != '\t' && *p != '\n' && i < 63) out[i++] = *p++;
    out[i] = '\0';
}

}  // namespace

extern "C" {

int LBM_LoadOBJ(const char *path, LBMModel *model) {
    if (!path || !model) return 0;
    memset(model, 0, sizeof(*model));
    const int nv = count_lines_with(path, 'v');
    const int nf = count_lines_with(path, 'f');
    if (nv < 0 || nf < 0) return 0;
    model->vertices = (float *)calloc((size_t)(nv > 0 ? nv : 1) * 3, sizeof(float));
    model->faces = (int *)calloc((size_t)(nf > 0 ? nf : 1) * 3, sizeof(int));
    if (!model->vertices || !model->faces) {
        LBM_FreeModel(model);
        return 0;
    }
    FILE *f = fopen(path, "r");
    if (!f) {
        LBM_FreeModel(model);
        return 0;
    }
    // model_loader.c:80-137: only the first three vertex references of a
    // face are kept, so quads and larger polygons are truncated
    char line[512];
    int vi = 0, fi = 0;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == 'v' && line[1] == ' ' && vi < nv) {
            sscanf(line, "v %f %f %f", &model->vertices[3 * vi], &model->vertices[3 * vi + 1],
                   &model->vertices[3 * vi + 2]);
            vi++;
        } else if (line[0] == 'f' && line[1] == ' ' && fi < nf) {
            char a[64] = {0}, b[64] = {0}, c[64] = {0};
            char *p = line + 2;
            while (*p == ' ' || *p == '\t') p++;
            read_token(p, a);
            while (*p == ' ' || *p == '\t') p++;
            read_token(p, b);
            while (*p == ' ' || *p == '\t') p++;
            read_token(p, c);
            model->faces[3 * fi] = parse_index(a);
            model->faces[3 * fi + 1] = parse_index(b);
            model->faces[3 * fi + 2] = parse_index(c);
            fi++;
        }
    }
    fclose(f);
    model->vertexCount = nv;
    model->faceCount = fi;
    return 1;
}

void LBM_FreeModel(LBMModel *model) {
    if (!model) return;
    free(model->vertices);
    free(model->faces);
    memset(model, 0, sizeof(*model));
}

int LBM_ModelBounds(const LBMModel *model, float scale, float offsetX, float offsetY,
                    float offsetZ, float rotationY, float *bounds9) {
    if (!bounds9) return 0;
    // model_bounds.c:154-160
    if (!model || model->vertexCount == 0) {
        bounds9[0] = bounds9[1] = bounds9[2] = -0.5f;
        bounds9[3] = bounds9[4] = bounds9[5] = 0.5f;
        bounds9[6] = bounds9[7] = bounds9[8] = 0.0f;
        return 1;
    }
    const float radY = rotationY * M_PI / 180.0f;  // double intermediate, as the reference
    const float cosY = cosf(radY), sinY = sinf(radY);
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < model->vertexCount; i++) {
        const float x = model->vertices[3 * i] * scale + offsetX;
        const float y = model->vertices[3 * i + 1] * scale + offsetY;
        const float z = model->vertices[3 * i + 2] * scale + offsetZ;
        const float rx = x * cosY - z * sinY;
        const float rz = x * sinY + z * cosY;
        if (rx < mn[0]) mn[0] = rx;
        if (y < mn[1]) mn[1] = y;
        if (rz < mn[2]) mn[2] = rz;
        if (rx > mx[0]) mx[0] = rx;
        if (y > mx[1]) mx[1] = y;
        if (rz > mx[2]) mx[2] = rz;
    }
    for (int k = 0; k < 3; k++) {
        bounds9[k] = mn[k];
        bounds9[3 + k] = mx[k];
        bounds9[6 + k] = (mn[k] + mx[k]) * 0.5f;
    }
    return 1;
}

float *LBM_CreateTriangleBuffer(const LBMModel *model, float scale, float offsetX, float offsetY,
                                float offsetZ, float rotationY, int *outCount) {
    if (outCount) *outCount = 0;
    if (!model || model->faceCount == 0 || model->vertexCount == 0 || !outCount) return nullptr;
    float *tris = (float *)malloc((size_t)model->faceCount * 12 * sizeof(float));
    if (!tris) return nullptr;
    const float radY = rotationY * M_PI / 180.0f;
    const float cosY = cosf(radY), sinY = sinf(radY);
    int valid = 0;
    for (int i = 0; i < model->faceCount; i++) {
        // model_bounds.c:239-281: 1-based indices, faces with an index out of
        // range are skipped
        const int idx[3] = {model->faces[3 * i] - 1, model->faces[3 * i + 1] - 1,
                            model->faces[3 * i + 2] - 1};
        bool ok = true;
        for (int k = 0; k < 3; k++) ok = ok && idx[k] >= 0 && idx[k] < model->vertexCount;
        if (!ok) continue;
        float *t = tris + 12 * (size_t)valid;
        for (int k = 0; k < 3; k++) {
            const float *v = model->vertices + 3 * idx[k];
            const float x = v[0] * scale + offsetX;
            const float y = v[1] * scale + offsetY;
            const float z = v[2] * scale + offsetZ;
            t[4 * k + 0] = x * cosY - z * sinY;
            t[4 * k + 1] = y;
            t[4 * k + 2] = x * sinY + z * cosY;
            t[4 * k + 3] = 0.0f;
        }
        valid++;
    }
    *outCount = valid;
    return tris;
}

void LBM_FreeTriangles(float *triangles) { free(triangles); }

int LBM_PlaceModel(const LBMModel *model, float scaleOrZero, float *scale, float *offset3,
                   float *rotationY) {
    if (!model || !scale || !offset3 || !rotationY || model->vertexCount == 0) return 0;
    // main.c:251-307: raw bounds, auto scale 2.4 / max dimension, centre
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < model->vertexCount; i++)
        for (int k = 0; k < 3; k++) {
            const float v = model->vertices[3 * i + k];
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
        }
    float c[3];
    for (int k = 0; k < 3; k++) c[k] = (mn[k] + mx[k]) * 0.5f;
    const float maxDim = fmaxf(mx[0] - mn[0], fmaxf(mx[1] - mn[1], mx[2] - mn[2]));
    const float s = scaleOrZero > 0.0f ? scaleOrZero : 2.4f / maxDim;
    float off[3] = {-c[0] * s, -c[1] * s, -c[2] * s};
    // main.c:312-339: rotate 90 degrees about y when z is the longest
    // horizontal extent
    float mnX = FLT_MAX, mxX = -FLT_MAX, mnZ = FLT_MAX, mxZ = -FLT_MAX;
    for (int i = 0; i < model->vertexCount; i++) {
        const float x = model->vertices[3 * i] * s + off[0];
        const float z = model->vertices[3 * i + 2] * s + off[2];
        if (x < mnX) mnX = x;
        if (x > mxX) mxX = x;
        if (z < mnZ) mnZ = z;
        if (z > mxZ) mxZ = z;
    }
    const float rot = (mxZ - mnZ > mxX - mnX) ? 90.0f : 0.0f;
    // main.c:341-349: centre at world x = -2 after the rotation
    const float radY = rot * (float)M_PI / 180.0f;
    off[0] += -2.0f * cosf(radY);
    off[2] += 2.0f * sinf(radY);
    *scale = s;
    offset3[0] = off[0];
    offset3[1] = off[1];
    offset3[2] = off[2];
    *rotationY = rot;
    return 1;
}

int LBM_ReynoldsToTau(float latticeVelocity, float charLength, float reynolds, float *tau,
                      float *viscosity, float *effectiveReynolds) {
    if (!tau || !viscosity || !effectiveReynolds || reynolds <= 0.0f) return 0;
    // main.c:447-460: nu = U L / Re, tau = 3 nu + 1/2, clamped at 0.52
    float nu = (latticeVelocity * charLength) / reynolds;
    float t = 3.0f * nu + 0.5f;
    float re = reynolds;
    int capped = 0;
    if (t < 0.52f) {
        nu = (0.52f - 0.5f) / 3.0f;
        t = 0.52f;
        re = (latticeVelocity * charLength) / nu;
        capped = 1;
    }
    *tau = t;
    *viscosity = nu;
    *effectiveReynolds = re;
    return capped ? 2 : 1;
}

float LBM_Strouhal(const float *clSeries, int clCount, int lbmSubsteps, int sampleInterval,
                   float charLength, float latticeVelocity, float *peakFrequency) {
    // drag_metrics.c:8-68: discard the first 35 %, remove the mean, Hann
    // window, one-sided DFT without DC, St = f_peak L / U
    if (peakFrequency) *peakFrequency = 0.0f;
    if (!clSeries || clCount < 12) return 0.0f;
    const int start = clCount * 35 / 100;
    const int n = clCount - start;
    const float *sig = clSeries + start;
    float mean = 0;
    for (int i = 0; i < n; i++) mean += sig[i];
    mean /= n;
    float *win = (float *)malloc(n * sizeof(float));
    if (!win) return 0.0f;
    for (int i = 0; i < n; i++) {
        const float w = 0.5f * (1.0f - cosf(2.0f * (float)M_PI * i / (n - 1)));
        win[i] = (sig[i] - mean) * w;
    }
    const float fs = 1.0f / (sampleInterval * lbmSubsteps);
    const int nfreqs = n / 2;
    float peakPow = 0, peakFreq = 0;
    for (int k = 1; k < nfreqs; k++) {
        float re = 0, im = 0;
        for (int i = 0; i < n; i++) {
            const float angle = 2.0f * (float)M_PI * k * i / n;
            re += win[i] * cosf(angle);
            im -= win[i] * sinf(angle);
        }
        const float pw = re * re + im * im;
        if (pw > peakPow) {
            peakPow = pw;
            peakFreq = (float)k * fs / n;
        }
    }
    free(win);
    if (peakFrequency) *peakFrequency = peakFreq;
    return (latticeVelocity > 1e-10f) ? peakFreq * charLength / latticeVelocity : 0;
}

}  // extern "C"
