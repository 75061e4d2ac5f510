// yspec_main.cpp -- the `yspec input.in` command (yspec.f90:1-511) on the
// B200 engine: same argument, parameter file, model deck and per-receiver
// ASCII output files as the reference.  Set YSPEC_DEVICE to pick the GPU.
#include <cstdio>
#include <cstdlib>

#include "yspec_host.h"

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: yspec input.in\n");
        return 2;
    }
    const char* dev = std::getenv("YSPEC_DEVICE");
    int rc = ysh_run(argv[1], dev ? std::atoi(dev) : 0, 1, nullptr, nullptr, nullptr);
    if (rc) {
        std::fprintf(stderr, "%s\n", ysh_status_string(rc));
        return 1;
    }
    return 0;
}
