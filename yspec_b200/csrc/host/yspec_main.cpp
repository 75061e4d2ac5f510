// yspec_main.cpp -- the `yspec input.in` command (yspec.f90:1-511) on the
// B200 engine: same argument, parameter file, model deck and per-receiver
// ASCII output files as the reference.  Set YSPEC_DEVICE to pick the GPU.
// `yspec a.in b.in ...` runs several events; those sharing a model deck
// are solved as one batch (each still writes its own files).  With
// YSPEC_TIMING set, a single-event run reports the wall time of its set-up,
// engine and writer phases on stderr.  `yspec --potential input.in` writes
// the potential traces instead (prefix.pot.1 .. prefix.pot.nr: time and the
// gravitational potential perturbation at each receiver).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "yspec_host.h"

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: yspec input.in [more.in ...] | yspec --potential input.in\n");
        return 2;
    }
    const char* dev = std::getenv("YSPEC_DEVICE");
    const int device = dev ? std::atoi(dev) : 0;
    if (std::strcmp(argv[1], "--potential") == 0) {
        if (argc != 3) {
            std::fprintf(stderr, "usage: yspec --potential input.in\n");
            return 2;
        }
        int rc = ysh_run_potential(argv[2], device, 1, nullptr, nullptr, nullptr);
        if (rc) {
            std::fprintf(stderr, "%s\n", ysh_status_string(rc));
            return 1;
        }
        return 0;
    }
    if (argc == 2) {
        int rc = ysh_run(argv[1], device, 1, nullptr, nullptr, nullptr);
        if (rc) {
            std::fprintf(stderr, "%s\n", ysh_status_string(rc));
            return 1;
        }
        return 0;
    }
    int failed = -1;
    int rc = ysh_run_batch(argc - 1, argv + 1, device, 1, &failed);
    if (rc) {
        if (failed >= 0) std::fprintf(stderr, "%s: ", argv[1 + failed]);
        std::fprintf(stderr, "%s\n", ysh_status_string(rc));
        return 1;
    }
    return 0;
}
