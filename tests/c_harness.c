/* A plain C99 caller of libtopgpu.so's host-side ABI (include/topgpu.h), the
 * way a MATLAB MEX gateway or a C application would bind it: version, mesh
 * model with the built-in cantilever BCs, its sizes and arrays (including the
 * error path of a too-small buffer), and, given a path, a .TopVoxel model.
 * Prints one JSON object; exit status 0 when every call behaved. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "topgpu.h"

static int fail(const char *what, int st)
{
    fprintf(stderr, "%s: status %d: %s\n", what, st, top_last_error());
    return 1;
}

int main(int argc, char **argv)
{
    const int ny = 8, nx = 16, nz = 8;
    uint8_t *mask = malloc((size_t)ny * nx * nz);
    if (!mask) return 1;
    memset(mask, 1, (size_t)ny * nx * nz);
    top_mesh *m = NULL;
    int st = top_mesh_create(mask, ny, nx, nz, 20000, 0.3, 1.0 / nx, 0, &m);
    free(mask);
    if (st != TOP_OK) return fail("top_mesh_create", st);
    if ((st = top_mesh_apply_optcase(m, 1)) != TOP_OK) return fail("top_mesh_apply_optcase", st);
    int64_t info[1 + 8 * 8];
    if ((st = top_mesh_info(m, info, 1 + 8 * 8)) != TOP_OK) return fail("top_mesh_info", st);
    int64_t nFix = 0, nF = 0, nEmb = 0;
    if ((st = top_mesh_get(m, 0, "fixingCond", NULL, 0, &nFix)) != TOP_OK) return fail("fixingCond", st);
    if ((st = top_mesh_get(m, 0, "F", NULL, 0, &nF)) != TOP_OK) return fail("F", st);
    if ((st = top_mesh_get(m, 0, "eleMapBack", NULL, 0, &nEmb)) != TOP_OK) return fail("eleMapBack", st);
    double *F = malloc(sizeof(double) * (size_t)nF);
    if (!F) return 1;
    if ((st = top_mesh_get(m, 0, "F", F, nF, NULL)) != TOP_OK) return fail("F copy", st);
    double fsum = 0;
    for (int64_t i = 0; i < nF; ++i) fsum += F[i];
    /* a buffer one element short must be refused with TOP_ERR_SHAPE and a message */
    const int small = top_mesh_get(m, 0, "F", F, nF - 1, NULL);
    const int smallOk = small == TOP_ERR_SHAPE && strlen(top_last_error()) > 0;
    const int unknown = top_mesh_get(m, 0, "noSuchArray", NULL, 0, NULL);
    free(F);
    printf("{\"version\": %d, \"levels\": %lld, \"Ne\": %lld, \"Nn\": %lld, \"nFix\": %lld, \"nF\": %lld, "
           "\"nEleMapBack\": %lld, \"Fsum\": %.17g, \"smallBufferRefused\": %d, \"unknownName\": %d",
           top_version(), (long long)info[0], (long long)info[1 + 4], (long long)info[1 + 5], (long long)nFix,
           (long long)nF, (long long)nEmb, fsum, smallOk, unknown);
    top_mesh_destroy(m);
    if (argc > 1) {
        top_mesh *f = NULL;
        if ((st = top_mesh_create_from_topvoxel(argv[1], 20000, 0.3, &f)) != TOP_OK) return fail("topvoxel", st);
        int64_t nPassive = 0, res[3] = {0, 0, 0}, nRes = 0;
        int32_t r32[3];
        if ((st = top_mesh_get(f, 0, "passiveElements", NULL, 0, &nPassive)) != TOP_OK) return fail("passive", st);
        if ((st = top_mesh_get(f, 0, "resolution", r32, 3, &nRes)) != TOP_OK) return fail("resolution", st);
        for (int k = 0; k < 3; ++k) res[k] = r32[k];
        printf(", \"file\": {\"nPassive\": %lld, \"resolution\": [%lld, %lld, %lld]}", (long long)nPassive,
               (long long)res[0], (long long)res[1], (long long)res[2]);
        top_mesh_destroy(f);
    }
    printf("}\n");
    return 0;
}
