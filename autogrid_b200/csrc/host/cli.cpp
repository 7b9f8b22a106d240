// autogrid4_b200: command-line drop-in for `autogrid4 -p file.gpf -l file.glg`
// (setflags.cpp:36-194): parse the GPF, compute the maps on the GPU, write the
// map files.  Exit status 0 on "Successful Completion", 1 otherwise.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "autogrid_b200.h"

static const char *kHelp =
    "\t-p parameter_filename\n\t\t\t-l log_filename\n\t\t\t-d (increment debug level)\n"
    "\t\t\t-h (display this message)\n\t\t\t--version (print version information)\n"
    "\t\t\t--fp64 (FP64 twin instead of the FP32 production path)\n\t\t\t--device N\n"
    "\t\t\t--host-writer (format the map files on the host instead of the GPU)\n";

int main(int argc, char **argv)
{
    std::string gpf, glg;
    int device = 0;
    bool fp64 = false, host_writer = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "-p" && i + 1 < argc) gpf = argv[++i];
        else if (a == "-l" && i + 1 < argc) glg = argv[++i];
        else if (a == "-d") {}
        else if (a == "-h" || a == "-u") { std::printf("usage: AutoGrid %s\n", kHelp); return 0; }
        else if (a == "--version" || a == "-v") {
            std::printf("AutoGrid-B200 4.2.7.x (AutoGrid 4 grid maps on NVIDIA B200, ABI %d)\n", ag_abi_version());
            return 0;
        }
        else if (a == "--fp64") fp64 = true;
        else if (a == "--host-writer") host_writer = true;
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else { std::fprintf(stderr, "%s: unknown switch %s\n", argv[0], a.c_str()); return 1; }
    }
    if (gpf.empty()) {
        std::fprintf(stderr, "%s: -p parameter_filename is required\n\t%s", argv[0], kHelp);
        return 1;
    }
    ag_job *job = nullptr;
    ag_status st = ag_job_load(gpf.c_str(), glg.empty() ? nullptr : glg.c_str(), &job);
    if (st != AG_OK) {
        std::fprintf(stderr, "\n%s: ERROR: %s\n\n%s: Unsuccessful Completion.\n", argv[0], ag_last_error(), argv[0]);
        return 1;
    }
    const ag_problem *p = ag_job_problem(job);
    ag_context *ctx = nullptr;
    st = ag_context_create(device, &ctx);
    const size_t P = (size_t)p->n1[0] * p->n1[1] * p->n1[2];
    const size_t n_out = (size_t)p->n_maps + (p->floating_grid ? 1 : 0) + (p->constriction_grid ? 1 : 0);
    if (st == AG_OK) {
        ag_opts o{};
        o.precision = fp64 ? AG_PREC_FP64 : AG_PREC_FP32;
        if (!host_writer) {
            // maps stay on the device; their text is formatted there
            const char *text = nullptr;
            std::vector<size_t> bytes(n_out);
            std::vector<double> emin((size_t)p->n_maps + 1), emax((size_t)p->n_maps + 1);
            st = ag_maps_compute_text(ctx, p, &o, &text, bytes.data(), emin.data(), emax.data());
            if (st == AG_OK) st = ag_job_write_text(job, text, bytes.data(), emin.data(), emax.data());
        } else if (fp64) {
            std::vector<double> maps(n_out * P);
            st = ag_maps_compute_f64(ctx, p, &o, maps.data());
            if (st == AG_OK) st = ag_job_write_maps_f64(job, maps.data());
        } else {
            std::vector<float> maps(n_out * P);
            st = ag_maps_compute(ctx, p, &o, maps.data());
            if (st == AG_OK) st = ag_job_write_maps_f32(job, maps.data());
        }
    }
    if (st != AG_OK) {
        const std::string msg = ag_last_error();
        ag_job_fail(job, msg.c_str());
        std::fprintf(stderr, "\n%s: ERROR: %s\n\n%s: Unsuccessful Completion.\n", argv[0], msg.c_str(), argv[0]);
    }
    ag_context_destroy(ctx);
    ag_job_free(job);
    return st == AG_OK ? 0 : 1;
}
