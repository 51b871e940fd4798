// LAMMPS input-script front end for the USER-MESO mDPD/DPD path: the commands a deck for
// atom_style mdpd/atomic/meso or dpd/atomic/meso, pair_style mdpd/meso or dpd/meso,
// fix nve/meso, fix aboundary/rho/meso, fix addforce/meso, fix density/meso and
// run_style mvv/meso uses, parsed with the reference's argument order and errors.
#pragma once

#include <map>
#include <stdexcept>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"

namespace mdpd {

class ScriptError : public std::runtime_error {
public:
    int code;
    ScriptError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

struct Region {
    double lo[3], hi[3];
};

struct DensityFix {
    std::string id, output;
    int group = 1, along = 0, nbin = 0, every = 0, window = 0;
    long long last_dump = -1;
    int frames = 0;
    std::vector<unsigned long long> counts;
    unsigned long long *d_counts = nullptr;
};

struct DumpSpec {
    std::string id, file;
    int group = 1, every = 1;
    std::vector<std::string> cols;
};

class Script {
public:
    explicit Script(int device = 0);
    ~Script();
    void command(const std::string &line);
    void file(const std::string &path);
    void run(long long n);
    void setup();                  // LAMMPS run setup (rebuild, density, force)
    std::string log;               // thermo + messages
    int echo = 0;

    // state access for the C ABI
    Box *box() { return box_.get(); }
    Batch *batch() { return batch_.get(); }
    const Spec &spec() const { return spec_; }
    Particles &particles() { return parts_; }
    long long step() const { return step_; }
    void thermo(Thermo &t);
    void sync_host();              // device state -> parts_ (tag order)
    void invalidate() { dirty_ = true; }
    StepConfig cfg;

private:
    std::map<std::string, std::string> vars_;
    std::map<std::string, Region> regions_;
    std::map<std::string, int> groups_;  // name -> bit index
    int ngroup_ = 1;
    Spec spec_;
    Particles parts_;
    bool box_defined_ = false;
    bool dirty_ = true;        // host state newer than device
    int thermo_every_ = 0;
    long long step_ = 0;
    double lattice_a_ = 1.0;
    int lattice_fcc_ = 0;
    int pair_set_ = 0;
    std::string nve_fix_, rho_fix_, ab_fix_;
    std::vector<DensityFix> dens_;
    std::vector<DumpSpec> dumps_;
    std::unique_ptr<Box> box_;
    std::unique_ptr<Batch> batch_;
    int device_ = 0;
    bool device_ready_ = false;

    std::string substitute(const std::string &line);
    double eval(const std::string &expr);
    double num(const std::string &tok);
    int inum(const std::string &tok);
    int group_bit(const std::string &name);
    void type_range(const std::string &tok, int &lo, int &hi);
    void ensure_device();
    void emit_thermo(bool header);
    void density_sample(long long step);
    void density_dump(DensityFix &d, long long stamp);
    void write_dump(const DumpSpec &d);
    void write_data(const std::string &path);
    void read_data(const std::string &path);
    void add_atom(int type, const double *x);
};

}  // namespace mdpd
