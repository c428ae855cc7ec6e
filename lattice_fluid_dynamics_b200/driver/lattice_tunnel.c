/*
 * lattice_tunnel -- headless wind-tunnel executable over liblattice_lbm.so.
 *
 * Accepts the reference binary's options (simulation/src/cli.c:12-181) so
 * that scripts driving it (simulation/modal_worker.py:370-385,
 * simulation/test/benchmark.sh:47-51) can call this one instead; the
 * solver loop and its stdout lines are LBM_TunnelRun's.  Options that only
 * concern rendering (--viz, --collision, --output) are accepted and
 * ignored; --superres is not available.  Extensions: --substeps=N
 * (lattice steps per frame, default 10), --storage=fp32|fp16|bf16|fp64,
 * --log=PATH.
 */
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lattice_lbm.h"

static void usage(const char *argv0) {
    printf("Usage: %s [options]\n", argv0);
    printf("Options:\n");
    printf("  -w, --wind=SPEED      Wind speed 0-5 (default: 1.0)\n");
    printf("  -d, --duration=SECS   Output duration at 60 frames/s (required, > 0)\n");
    printf("  -m, --model=PATH      Path to OBJ model file\n");
    printf("  -a, --angle=DEGREES   Ahmed body slant angle (25 or 35)\n");
    printf("  -s, --scale=SCALE     Model scale factor (default: auto)\n");
    printf("  -r, --reynolds=RE     Target Reynolds number (0=derive from wind speed)\n");
    printf("  -g, --grid=XxYxZ      Grid size (default: 128x64x64)\n");
    printf("  -S, --smagorinsky=CS  Smagorinsky constant 0-0.5 (default: 0.1)\n");
    printf("  -M, --mrt             MRT collision (always on)\n");
    printf("  --vtk-output=PATH     Directory for VTK field dumps\n");
    printf("  --vtk-interval=N      Frames between VTK dumps (default: 100)\n");
    printf("  --substeps=N          Lattice steps per frame (default: 10)\n");
    printf("  --storage=TYPE        fp32 (default), fp16, bf16 or fp64 populations\n");
    printf("  --log=PATH            Write the run's lines to PATH instead of stdout\n");
    printf("  -v, -c, -o            Accepted for compatibility; nothing is rendered\n");
    printf("  -h, --help            Show this help\n");
}

int main(int argc, char *argv[]) {
    LBMTunnelOptions o;
    LBM_TunnelDefaults(&o);
    static char modelPath[512] = "assets/3d-files/car-model.obj";
    static char vtkPath[256] = "";
    static char logPath[512] = "";
    static struct option longopts[] = {
        {"wind", required_argument, 0, 'w'},       {"viz", required_argument, 0, 'v'},
        {"collision", required_argument, 0, 'c'},  {"duration", required_argument, 0, 'd'},
        {"output", required_argument, 0, 'o'},     {"model", required_argument, 0, 'm'},
        {"angle", required_argument, 0, 'a'},      {"scale", required_argument, 0, 's'},
        {"reynolds", required_argument, 0, 'r'},   {"grid", required_argument, 0, 'g'},
        {"smagorinsky", required_argument, 0, 'S'}, {"mrt", no_argument, 0, 'M'},
        {"vtk-output", required_argument, 0, 'V'}, {"vtk-interval", required_argument, 0, 'I'},
        {"superres", no_argument, 0, 'R'},         {"sr-weights", required_argument, 0, 'W'},
        {"substeps", required_argument, 0, 'N'},   {"storage", required_argument, 0, 'T'},
        {"log", required_argument, 0, 'L'},        {"help", no_argument, 0, 'h'},
        {0, 0, 0, 0}};
    int c;
    while ((c = getopt_long(argc, argv, "w:v:c:d:o:m:a:r:s:g:S:Mh", longopts, NULL)) != -1) {
        switch (c) {
        case 'w':
            o.windSpeed = (float)atof(optarg);
            if (o.windSpeed < 0) o.windSpeed = 0;
            if (o.windSpeed > 5) o.windSpeed = 5;
            break;
        case 'v':
        case 'c':
        case 'o':
        case 'W':
        case 'M':
            break;
        case 'd':
            o.renderDuration = atoi(optarg);
            if (o.renderDuration < 0) o.renderDuration = 0;
            break;
        case 'm':
            strncpy(modelPath, optarg, sizeof(modelPath) - 1);
            break;
        case 'a': {
            const int a = atoi(optarg);
            if (a == 25 || a == 35)
                snprintf(modelPath, sizeof(modelPath), "assets/3d-files/ahmed_%ddeg_m.obj", a);
            break;
        }
        case 's':
            o.scale = (float)atof(optarg);
            break;
        case 'r':
            o.reynolds = (float)atof(optarg);
            if (o.reynolds < 0) o.reynolds = 0;
            break;
        case 'S':
            o.smagorinskyCs = (float)atof(optarg);
            if (o.smagorinskyCs < 0.0f) o.smagorinskyCs = 0.0f;
            if (o.smagorinskyCs > 0.5f) o.smagorinskyCs = 0.5f;
            break;
        case 'g':
            if (sscanf(optarg, "%dx%dx%d", &o.gridX, &o.gridY, &o.gridZ) != 3) {
                const int n = atoi(optarg);
                if (n > 0) {
                    o.gridX = n;
                    o.gridY = n / 2;
                    o.gridZ = n / 2;
                }
            }
            break;
        case 'V':
            strncpy(vtkPath, optarg, sizeof(vtkPath) - 1);
            break;
        case 'I':
            o.vtkInterval = atoi(optarg);
            if (o.vtkInterval < 1) o.vtkInterval = 1;
            break;
        case 'R':
            fprintf(stderr, "--superres is not available in this build; ignored\n");
            break;
        case 'N':
            o.substeps = atoi(optarg);
            if (o.substeps < 1) o.substeps = 1;
            break;
        case 'T':
            if (!strcmp(optarg, "fp32")) o.storage = LBM_STORAGE_FP32;
            else if (!strcmp(optarg, "fp16")) o.storage = LBM_STORAGE_FP16;
            else if (!strcmp(optarg, "bf16")) o.storage = LBM_STORAGE_BF16;
            else if (!strcmp(optarg, "fp64")) o.storage = LBM_STORAGE_FP64;
            else {
                fprintf(stderr, "unknown --storage=%s\n", optarg);
                return 2;
            }
            break;
        case 'L':
            strncpy(logPath, optarg, sizeof(logPath) - 1);
            break;
        case 'h':
        default:
            usage(argv[0]);
            return c == 'h' ? 0 : 2;
        }
    }
    if (o.renderDuration <= 0) {
        fprintf(stderr, "--duration must be > 0 (there is no interactive mode)\n");
        return 2;
    }
    o.modelPath = modelPath;
    o.vtkOutputPath = vtkPath;
    o.logPath = logPath;
    printf("Configuration:\n");
    printf("  Model: %s\n", modelPath);
    printf("  Wind Speed: %.1f m/s\n", o.windSpeed);
    if (o.reynolds > 0) printf("  Reynolds: %.0f\n", o.reynolds);
    printf("  Render Mode: %d seconds\n", o.renderDuration);
    fflush(stdout);
    LBMTunnelResult r;
    const int rc = LBM_TunnelRun(&o, &r);
    if (rc != LBM_OK) {
        fprintf(stderr, "lattice_tunnel: %s\n", LBM_GetErrorString(rc));
        return 1;
    }
    return 0;
}
