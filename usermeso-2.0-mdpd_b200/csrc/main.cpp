// lmp_mdpd: command-line driver, `lmp_mdpd -in script [-device N] [-echo]`, the
// single-process counterpart of the reference's `lmp_meso -in script -device N`
// (src/main.cpp:31-47, src/lammps.cpp:170-191); `lmp_mdpd -jobs spec.json [-out results.jsonl]`
// runs a JSON job spec on the serving loop and writes one JSON line per job.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/mdpd.h"

int main(int argc, char **argv)
{
    const char *in = nullptr, *jobs = nullptr, *out = nullptr;
    mdpd_opts o = {0, 0};
    for (int k = 1; k < argc; ++k) {
        if (!strcmp(argv[k], "-in") && k + 1 < argc) in = argv[++k];
        else if (!strcmp(argv[k], "-jobs") && k + 1 < argc) jobs = argv[++k];
        else if (!strcmp(argv[k], "-out") && k + 1 < argc) out = argv[++k];
        else if (!strcmp(argv[k], "-device") && k + 1 < argc) o.device = atoi(argv[++k]);
        else if (!strcmp(argv[k], "-echo")) o.verbose = 1;
    }
    if (jobs) {
        const int rc = mdpd_run_jobs(jobs, out, &o);
        if (rc) fprintf(stderr, "ERROR: %s\n", mdpd_last_error(nullptr));
        return rc;
    }
    if (!in) {
        fprintf(stderr, "usage: %s -in script [-device N] | -jobs spec.json [-out results.jsonl] [-device N]\n", argv[0]);
        return 2;
    }
    mdpd_t *h = nullptr;
    int rc = mdpd_create(&h, &o);
    if (rc) {
        fprintf(stderr, "ERROR: %s\n", mdpd_last_error(nullptr));
        return rc;
    }
    rc = mdpd_file(h, in);
    fputs(mdpd_log(h), stdout);
    if (rc) fprintf(stderr, "ERROR: %s\n", mdpd_last_error(h));
    mdpd_destroy(h);
    return rc;
}
