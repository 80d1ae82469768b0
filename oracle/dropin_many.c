/*
 * The drop-in's three stages run for several spectra in one process, as a
 * worker of the reference's pool (bin/accelsearch_pipeline_cu.py) runs them:
 * for each .fft file given after the flags, accelsearch_CPU1, accelsearch_GPU
 * and accelsearch_CPU2 (the sequence of src/accelsearch_cu.c:22-34).  Prints
 * each accelsearch_GPU call's wall time to stderr.
 *
 *     accelsearch_b200_many <flags...> -- a.fft b.fft ...
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "accel.h"

static double now(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

int main(int argc, char *argv[])
{
    int sep = 1;
    while (sep < argc && strcmp(argv[sep], "--"))
        sep++;
    if (sep >= argc - 1) {
        fprintf(stderr, "usage: %s <flags...> -- file.fft ...\n", argv[0]);
        return 2;
    }
    for (int f = sep + 1; f < argc; f++) {
        char *av[64];
        int ac = 0;
        for (int i = 0; i < sep && ac < 62; i++)
            av[ac++] = argv[i];
        av[ac++] = argv[f];
        av[ac] = NULL;
        subharminfo **subharminfs;
        accelobs obs;
        infodata idata;
        GSList *cands = NULL;
        Cmdline *cmd;
        accelsearch_CPU1(ac, av, &subharminfs, &obs, &idata, &cmd);
        const double t0 = now();
        const int rc = accelsearch_GPU(obs, subharminfs, &cands, cmd);
        fprintf(stderr, "accelsearch_GPU %s: %.3f s rc %d\n", argv[f], now() - t0, rc);
        accelsearch_CPU2(&cands, &obs, &idata, cmd);
    }
    return 0;
}
