/*
 * Entry point of the reference build used as an oracle (test infrastructure only).
 * Calls the reference's own run_simulation (source/run_simulation.cuh:60-63) with the
 * same command line the reference executable accepts (source/MAIN.cu:3-24) and
 * reports the wall-clock time of the whole call on stdout.
 */
#include "run_simulation.cuh"
#include <chrono>
#include <cstdio>

void ref_hooks_finish();

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        fprintf(stderr, "usage: %s [-epsilon e] [-solver hwfv1|mwdg2] [-dirroot d] case.par\n", argv[0]);
        return 2;
    }
    auto t0 = std::chrono::steady_clock::now();
    run_simulation(argc, argv);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    ref_hooks_finish();
    printf("REF_WALL_S %.6f\n", std::chrono::duration<double>(t1 - t0).count());
    return 0;
}
