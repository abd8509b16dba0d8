// ref_time -- test-only timing driver around the reference library (oracle/_ref).
//
// Times the reference's own electrostatics path in the only mode it computes
// (src/md/empole.cpp:96-357, empole_a: non-Ewald permanent multipoles over all
// pairs within the cutoff) through its public entry point, exactly as its
// `analyze` program sets it up (src/md/analyze.cpp:60-62: initial -> getcart ->
// mechanic) and then calls energy<CalcMode::Gradient>() (src/md/energy.cpp:31)
// `--reps` times.  initial() sets the OpenMP thread count to every processor
// it sees (src/md/initial.cpp:57-60); the driver reports that count.
// Prints one JSON object: n, nthread, em, a checksum of dem, and the
// seconds of each call.  The benchmark's CPU leg runs it beside the GPU; the
// product never runs it.
//
// usage: ref_time [--reps K] xyzfile -k keyfile

#include "action.h"
#include "atoms.h"
#include "calcMode.h"
#include "deriv.h"
#include "energi.h"
#include "energy.h"
#include "files.h"
#include "getcart.h"
#include "inform.h"
#include "initial.h"
#include "mechanic.h"
#include "openmp.h"
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace polmdqc;

int main(int argc, char** argv)
{
    int reps = 1;
    std::vector<char*> args;
    args.push_back((char*)"analyze");
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "--reps") && i + 1 < argc) { reps = atoi(argv[++i]); continue; }
        args.push_back(argv[i]);
    }
    if (reps < 1) reps = 1;
    args.push_back((char*)"e");
    args.push_back(nullptr);
    test = true;
    auto t0 = std::chrono::steady_clock::now();
    initial((int)args.size() - 1, args.data());
    getcart(ffile);
    mechanic();
    auto t1 = std::chrono::steady_clock::now();
    std::vector<double> secs;
    for (int r = 0; r < reps; r++) {
        auto a = std::chrono::steady_clock::now();
        energy<CalcMode::Gradient>();
        auto b = std::chrono::steady_clock::now();
        secs.push_back(std::chrono::duration<double>(b - a).count());
    }
    double dsum = 0, dabs = 0;
    for (int i = 0; i < 3 * n; i++) {  // dem is stored flat, x y z per atom
        dsum += dem[i];
        dabs += std::fabs(dem[i]);
    }
    printf("{\"n\": %d, \"nthread\": %d, \"em\": %.17g, \"dem_sum\": %.17g, \"dem_abs_sum\": %.17g, "
           "\"setup_s\": %.6f, \"call_s\": [",
           n, nthread, em, dsum, dabs, std::chrono::duration<double>(t1 - t0).count());
    for (int r = 0; r < reps; r++) printf("%s%.6f", r ? ", " : "", secs[r]);
    printf("]}\n");
    return 0;
}
