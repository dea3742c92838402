// gpu-mwdg2 executable: same command line as the reference's (source/MAIN.cu:3-24,
// source/input/read_command_line_params.cpp:3-47) plus `-precision 32|64`.
#include "../../include/mwdg2.h"

#include <cstdio>

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        fprintf(stderr, "usage: %s [-epsilon e] [-solver hwfv1|mwdg2] [-dirroot d] [-precision 32|64] case.par\n", argv[0]);
        return 2;
    }
    const mwdg2_status st = mwdg2_run_simulation(argc, argv);
    if (st != MWDG2_OK)
    {
        fprintf(stderr, "gpu-mwdg2: %s (status %d)\n", mwdg2_last_error(), (int)st);
        return 1;
    }
    return 0;
}
