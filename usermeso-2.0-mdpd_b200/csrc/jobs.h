// JSON job specs for the serving loop (jobs.cpp): a file of boxes to run, each a
// mdpd_box_spec with its step count, submitted to one server and reported as JSON lines.
#pragma once

#include <cstdint>
#include <ostream>
#include <string>
#include <vector>

#include "../../include/mdpd.h"

namespace mdpd {

struct JobEntry {
    std::string name;
    mdpd_job_spec spec{};
};

struct JobFile {
    uint64_t budget_bytes = 0;  // HBM admission budget of the server
    double timeout_s = 0.0;     // limit of the whole run (0: none)
    std::vector<JobEntry> jobs;
};

// read and check the file; throws std::runtime_error("PARSE: <path>: ...") naming the job and
// key at fault.  No device call.
JobFile read_job_file(const std::string &path);

// run every job on one server (opts: device), writing one JSON line per job in file order and
// a summary line to out; returns MDPD_OK or the MDPD_* code of the first job that did not
// finish (MDPD_ERR_TIMEOUT when the run hit timeout_s)
int run_job_file(const JobFile &jf, const mdpd_opts *opts, std::ostream &out);

}  // namespace mdpd
