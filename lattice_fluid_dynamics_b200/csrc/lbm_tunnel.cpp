// Headless wind-tunnel driver: the solver loop of the reference's main()
// with rendering, particles and the GL context left out.
//
// Reference behaviour restated here (simulation/src/main.c):
//   :438-465   Re from wind speed, Re -> viscosity -> tau with the 0.52 clamp
//   :471-553   grid set-up (mesh or AABB fallback, periodic y/z, Smagorinsky,
//              MRT, uniform inlet flow), effective Re, projected area and
//              blockage (Pope & Harper factor (1 - eps)^2)
//   :893-981   frame loop: inlet ramp over 300 frames, lbmSubsteps steps per
//              frame, VTI dumps, Cd start frame after ramp + 3 flow-throughs
//   :1249-1391 Cd / Cl / pressure-friction split every 20 frames, EMA,
//              convergence over the last 100 samples, auto-stop 120 frames on
//   :1404-1410 Strouhal number of the Cl series
// The printed lines keep the reference's formats (they are scraped by
// simulation/modal_worker.py:474-560 and simulation/test/benchmark.sh:57-79).
// Frames are not rendered; the loop ends when the reference's would with an
// output directory given (one output frame per frame from the start frame).
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <vector>

#include "../../include/lattice_lbm.h"

extern "C" {

void LBM_CdMonitorInit(LBMCdMonitor *m) {
    if (m) memset(m, 0, sizeof(*m));
}

int LBM_CdMonitorAdd(LBMCdMonitor *m, float cd, float cdCorr) {
    if (!m) return 0;
    // EMA seeded while no sample has been accepted into the history
    if (m->historyCount == 0) {
        m->ema = cdCorr;
    } else {
        const float alpha = 0.1f;
        m->ema = alpha * cdCorr + (1.0f - alpha) * m->ema;
    }
    if (!(cd > 0 && cd < 1000)) return 0;
    m->history[m->historyCount % LBM_CD_HISTORY_SIZE] = cd;
    m->historyCount++;
    if (m->historyCount < LBM_CD_HISTORY_SIZE || m->converged) return 0;
    float mean = 0;
    for (int j = 0; j < LBM_CD_HISTORY_SIZE; j++) mean += m->history[j];
    mean /= LBM_CD_HISTORY_SIZE;
    float var = 0;
    for (int j = 0; j < LBM_CD_HISTORY_SIZE; j++) {
        const float d = m->history[j] - mean;
        var += d * d;
    }
    const float relStd = sqrtf(var / LBM_CD_HISTORY_SIZE) / (mean + 1e-10f);
    if (relStd < 0.01f) {
        m->converged = 1;
        m->convergedMean = mean;
        m->convergedRelStd = relStd;
        return 1;
    }
    return 0;
}

void LBM_TunnelCoefficients(float fx, float fy, float px, float latticeVelocity, float refArea,
                            float blockageFactor, LBMCoefficients *out) {
    if (!out) return;
    const float rho0 = 1.0f;
    const float dynP = 0.5f * rho0 * latticeVelocity * latticeVelocity;
    const float denom = dynP * refArea;
    const bool ok = denom > 1e-10f;
    out->cd = ok ? fabsf(fx) / denom : 0.0f;
    out->cl = ok ? fy / denom : 0.0f;
    out->cdPressure = ok ? fabsf(px) / denom : 0.0f;
    out->cdFriction = out->cd - out->cdPressure;
    if (out->cdFriction < 0.0f) out->cdFriction = 0.0f;
    out->cdCorr = out->cd * blockageFactor;
}

int LBM_TunnelCdStartFrame(int sizeX, float latticeVelocity, int substeps, int maxFrames) {
    const int rampEnd = LBM_RAMP_FRAMES;
    const int flowThroughFrames = (int)(sizeX / (latticeVelocity * substeps * 2));
    int start = rampEnd + 3 * flowThroughFrames;
    if (maxFrames > 0 && start >= maxFrames) {
        start = maxFrames * 2 / 3;
        if (start < rampEnd && maxFrames > rampEnd) start = rampEnd;
    }
    return start;
}

float LBM_TunnelRampFactor(int frame) {
    return frame < LBM_RAMP_FRAMES ? (float)frame / (float)LBM_RAMP_FRAMES : 1.0f;
}

void LBM_TunnelDefaults(LBMTunnelOptions *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->windSpeed = 1.0f;
    o->gridX = 128;
    o->gridY = 64;
    o->gridZ = 64;
    o->smagorinskyCs = 0.1f;
    o->substeps = 10;
    o->latticeVelocity = 0.05f;
    o->vtkInterval = 100;
    o->storage = LBM_STORAGE_FP32;
}

int LBM_TunnelRun(const LBMTunnelOptions *opt, LBMTunnelResult *res) {
    if (!opt || !res || opt->renderDuration <= 0 || opt->substeps <= 0 || opt->gridX <= 0 ||
        opt->gridY <= 0 || opt->gridZ <= 0 || !(opt->latticeVelocity > 0.0f))
        return LBM_ERR_INVALID_ARGUMENT;
    memset(res, 0, sizeof(*res));
    FILE *out = stdout;
    if (opt->logPath && opt->logPath[0]) {
        out = fopen(opt->logPath, "w");
        if (!out) return LBM_ERR_INVALID_ARGUMENT;
    }
    const float U = opt->latticeVelocity;
    const int substeps = opt->substeps;

    // ---- model: load, place, bounds, triangles (main.c:240-366)
    LBMModel model;
    memset(&model, 0, sizeof(model));
    if (opt->modelPath && opt->modelPath[0]) LBM_LoadOBJ(opt->modelPath, &model);
    fprintf(out, "Model loaded: %d vertices, %d faces\n", model.vertexCount, model.faceCount);
    float scale = opt->scale > 0 ? opt->scale : 0.0f, off[3] = {0, 0, 0}, rotY = 0.0f;
    if (model.vertexCount > 0) {
        LBM_PlaceModel(&model, opt->scale > 0 ? opt->scale : 0.0f, &scale, off, &rotY);
        fprintf(out, "Auto scale: %.6f\n", scale);
        fprintf(out, "Auto-rotation: %d deg\n", (int)rotY);
    }
    float b[9];
    LBM_ModelBounds(&model, scale, off[0], off[1], off[2], rotY, b);
    fprintf(out,
            "Model bounds (rotated %.1f deg): min(%.2f, %.2f, %.2f) max(%.2f, %.2f, %.2f)\n",
            rotY, b[0], b[1], b[2], b[3], b[4], b[5]);
    int ntri = 0;
    float *tris = LBM_CreateTriangleBuffer(&model, scale, off[0], off[1], off[2], rotY, &ntri);
    fprintf(out, "Created %d valid triangles\n", ntri);
    res->triangles = ntri;

    // ---- Re -> tau (main.c:438-465)
    const float scaleX = opt->gridX / 8.0f;
    const float charLength = (b[3] - b[0]) * scaleX;
    float reynolds = opt->reynolds;
    if (reynolds <= 0) {
        reynolds = 200.0f * opt->windSpeed;
        if (reynolds < 50.0f) reynolds = 50.0f;
    }
    float tau = 0, nu = 0, reEff = 0;
    const int clamp = LBM_ReynoldsToTau(U, charLength, reynolds, &tau, &nu, &reEff);
    if (clamp == 2)
        fprintf(out, "  Re capped at %.0f (tau=%.2f needed for stable Cd, requested Re=%.0f)\n",
                reEff, tau, reynolds);
    reynolds = reEff;
    fprintf(out, "Reynolds number: %.0f\n", reynolds);
    fprintf(out, "  Char length: %.1f lattice units\n", charLength);
    fprintf(out, "  Viscosity: %.6f\n", nu);
    fprintf(out, "  tau: %.4f\n", tau);
    fprintf(out, "  CFL: %.4f\n", U);

    // ---- grid (main.c:471-553)
    fprintf(out, "Initializing LBM grid...\n");
    LBMGrid *grid = LBM_CreateEx(opt->gridX, opt->gridY, opt->gridZ, nu, opt->storage);
    if (!grid) {
        LBM_FreeTriangles(tris);
        LBM_FreeModel(&model);
        if (out != stdout) fclose(out);
        return LBM_ERR_OUT_OF_MEMORY;
    }
    fprintf(out, "LBM Grid: %dx%dx%d (%d cells), tau=%.3f\n", grid->sizeX, grid->sizeY,
            grid->sizeZ, grid->totalCells, grid->tau);
    if (tris && ntri > 0)
        LBM_SetSolidMesh(grid, tris, ntri, b[0], b[1], b[2], b[3], b[4], b[5]);
    else
        LBM_SetSolidAABB(grid, b[0], b[1], b[2], b[3], b[4], b[5]);
    {
        std::vector<int32_t> solid((size_t)grid->totalCells);
        LBM_CopySolid(grid, solid.data());
        int n = 0;
        for (int32_t s : solid) n += s == 1;
        res->solidCells = n;
        if (tris && ntri > 0) fprintf(out, "LBM mesh solid: %d cells marked as solid\n", n);
    }
    grid->periodicYZ = 1;
    grid->useSmagorinsky = 1;
    grid->smagorinskyCs = opt->smagorinskyCs;
    fprintf(out, "Smagorinsky SGS enabled (Cs=%.2f), periodic YZ\n", grid->smagorinskyCs);
    grid->useMRT = 1;
    fprintf(out, "MRT collision enabled\n");
    if (!LBM_InitializeFlow(grid, U, 0.0f, 0.0f)) {
        fprintf(stderr, "FATAL: LBM flow initialization failed\n");
        const int err = LBM_GetLastError(grid);
        LBM_Free(grid);
        LBM_FreeTriangles(tris);
        LBM_FreeModel(&model);
        if (out != stdout) fclose(out);
        return err != LBM_OK ? err : LBM_ERR_CUDA;
    }
    {
        const float sX = grid->sizeX / 8.0f;
        const float charL = (b[3] - b[0]) * sX;
        const float nuG = (grid->tau - 0.5f) / 3.0f;
        const float re = (nuG > 1e-10f) ? U * charL / nuG : 0;
        fprintf(out, "Effective Re = %.0f (U=%.3f, L=%.1f, nu=%.4f)\n", re, U, charL, nuG);
    }
    fprintf(out, "  Sample interval: %d lattice steps\n", substeps);
    const float sY = grid->sizeY / 4.0f, sZ = grid->sizeZ / 4.0f;
    const float bboxArea = (b[4] - b[1]) * sY * (b[5] - b[2]) * sZ;
    float refArea = LBM_ComputeProjectedArea(grid, 0);
    if (refArea < 1.0f) refArea = bboxArea;
    const float epsilon = refArea / ((float)grid->sizeY * grid->sizeZ);
    const float blockageFactor = (1.0f - epsilon) * (1.0f - epsilon);
    fprintf(out, "LBM initialized successfully\n");
    {
        const size_t cells = (size_t)grid->sizeX * grid->sizeY * grid->sizeZ;
        const size_t lbmBytes = cells * LBM_BytesPerUpdate(grid) + cells * 16 + cells * 4;
        fprintf(out, "  LBM buffers:      %.1f MB (%dx%dx%d grid)\n", lbmBytes / (1024.0 * 1024.0),
                grid->sizeX, grid->sizeY, grid->sizeZ);
        fprintf(out, "  Triangle mesh:    %.1f MB (%d triangles)\n",
                ntri * 48.0 / (1024.0 * 1024.0), ntri);
        fprintf(out, "  Total:            %.1f MB\n",
                (lbmBytes + ntri * 48.0) / (1024.0 * 1024.0));
    }
    fflush(out);
    res->tau = grid->tau;
    res->viscosity = nu;
    res->reynolds = reynolds;
    res->charLength = charLength;
    res->refArea = refArea;
    res->blockage = epsilon;
    res->blockageFactor = blockageFactor;

    // ---- frame loop (main.c:893-1391)
    int frame = 0, outputFrames = 0, maxFrames = opt->renderDuration * 60;
    LBMCdMonitor mon;
    LBM_CdMonitorInit(&mon);
    std::vector<float> cl;
    bool diagPrinted = false;
    const bool vtk = opt->vtkOutputPath && opt->vtkOutputPath[0];
    const int vtkInterval = opt->vtkInterval > 0 ? opt->vtkInterval : 1;
    cudaStream_t stream = (cudaStream_t)LBM_GetStream(grid);
    cudaStreamSynchronize(stream);
    const auto t0 = std::chrono::steady_clock::now();
    int status = LBM_OK;
    for (bool running = true; running;) {
        frame++;
        const float inlet = U * LBM_TunnelRampFactor(frame);
        LBM_StepN(grid, substeps, inlet, 0.0f, 0.0f);
        if (vtk && frame % vtkInterval == 0) writeVTI(grid, opt->vtkOutputPath, frame);
        const int cdStart = LBM_TunnelCdStartFrame(grid->sizeX, U, substeps, maxFrames);
        res->cdStartFrame = cdStart;
        const bool skip = frame < cdStart;
        if (frame >= cdStart && frame % LBM_CD_SAMPLE_INTERVAL == 0) {
            float fx, fy, fz, px, py, pz;
            LBM_ComputeDragForceDecomposed(grid, &fx, &fy, &fz, &px, &py, &pz);
            LBMCoefficients c;
            LBM_TunnelCoefficients(fx, fy, px, U, refArea, blockageFactor, &c);
            if (!diagPrinted) {
                const float bodyY = (b[4] - b[1]) * sY, bodyZ = (b[5] - b[2]) * sZ;
                fprintf(out, "  Cd calculation breakdown:\n");
                fprintf(out, "    Re = %.0f, U_lattice = %.4f, rho_0 = %.1f\n", reynolds, U, 1.0f);
                fprintf(out, "    Body (lattice): %.1f x %.1f x %.1f cells\n", charLength, bodyY,
                        bodyZ);
                fprintf(out, "    Projected area = %.1f cells^2 (bbox = %.1f)\n", refArea,
                        bboxArea);
                fprintf(out, "    Blockage = %.1f%%, correction = %.3f (Pope & Harper 1966)\n",
                        epsilon * 100.0f, blockageFactor);
                if (fminf(bodyY, bodyZ) < 10.0f)
                    fprintf(out, "    WARNING: body < 10 cells across -- Cd is unreliable at "
                                 "this resolution\n");
                if (epsilon > 0.05f)
                    fprintf(out, "    WARNING: blockage > 5%% -- confinement inflates Cd\n");
                diagPrinted = true;
            }
            // the EMA is updated before the history, as in the reference
            const int newlyConverged = LBM_CdMonitorAdd(&mon, c.cd, c.cdCorr);
            const int totalSteps = frame * substeps;
            const float tStar = charLength > 0 ? (float)totalSteps * U / charLength : 0.0f;
            const float flowThroughs =
                grid->sizeX > 0 ? (float)totalSteps * U / grid->sizeX : 0.0f;
            fprintf(out,
                    "  Drag Force: (%.4f, %.4f, %.4f), Cd=%.3f Cd_corr=%.3f Cl=%.3f (avg=%.3f) "
                    "t*=%.3f flow-throughs=%.2f\n",
                    fx, fy, fz, c.cd, c.cdCorr, c.cl, mon.ema, tStar, flowThroughs);
            fprintf(out, "  Cd_pressure=%.3f Cd_friction=%.3f\n", c.cdPressure, c.cdFriction);
            fflush(out);
            cl.push_back(c.cl);
            res->cdSamples++;
            res->lastCd = c.cd;
            res->lastCdCorr = c.cdCorr;
            res->lastCl = c.cl;
            if (newlyConverged) {
                fprintf(out, "  Cd converged (mean=%.3f, relStd=%.4f)\n", mon.convergedMean,
                        mon.convergedRelStd);
                const int extra = 120;
                if (outputFrames + extra < maxFrames) maxFrames = outputFrames + extra;
            }
            if (LBM_GetLastError(grid) != LBM_OK) {
                status = LBM_GetLastError(grid);
                running = false;
            }
        }
        if (outputFrames >= maxFrames) {
            fprintf(out, "Render complete: %d frames\n", outputFrames);
            running = false;
        }
        if (!skip) outputFrames++;
    }
    cudaStreamSynchronize(stream);
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->frames = frame;
    res->latticeSteps = (long long)frame * substeps;
    res->seconds = secs;
    res->mlups = secs > 0 ? (double)res->latticeSteps * grid->totalCells / secs / 1e6 : 0.0;
    res->cdEma = mon.ema;
    res->converged = mon.converged;
    res->convergedMean = mon.convergedMean;

    // ---- Strouhal (main.c:1404-1410, drag_metrics.c:8-68)
    float f = 0;
    const float st = LBM_Strouhal(cl.data(), (int)cl.size(), substeps, LBM_CD_SAMPLE_INTERVAL,
                                  charLength, U, &f);
    if (cl.size() >= 12)
        fprintf(out, "St=%.4f (f=%.6f, L=%.1f, U=%.3f)\n", st, f, charLength, U);
    res->strouhal = st;
    res->sheddingFrequency = f;
    fprintf(out, "Tunnel: %d frames, %lld lattice steps, %.3f s, %.1f MLUPS\n", res->frames,
            res->latticeSteps, res->seconds, res->mlups);
    fflush(out);
    if (out != stdout) fclose(out);
    LBM_Free(grid);
    LBM_FreeTriangles(tris);
    LBM_FreeModel(&model);
    return status;
}

}  // extern "C"
