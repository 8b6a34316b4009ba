// miniafqmc - the miniapp's driver program over the C ABI of libafqmc_b200.
//
// Restates the main program of QMCPACK miniAFQMC (src/miniapps/miniafqmc_base.cpp:93-360)
// with its flags, set-up, substep loop and output, calling the B200 library's operations
// (include/afqmc_b200.h) where the reference calls its afqmc_sys / base:: templates:
//
//   Initialize from the input file          miniafqmc_base.cpp:174-180
//   half-rotation of Spvn (-t yes)          :181-185   -> afq_halfrotate (GPU)
//   walkers = conj(trial), weights 1        :226-236   -> afq_set_walkers
//   initial density matrix + energy         :239-240
//   per substep: DM, vbias, X, vHS,         :251-328   -> afq_mixed_density_matrix,
//     propagate, overlaps, weights                        afq_vbias, afq_sigma, afq_vhs,
//                                                         afq_propagate, afq_overlaps,
//                                                         afq_update_weights
//   orthogonalisation every northo          :330-337   -> afq_orthogonalize, afq_overlaps
//   energy after each step, printed         :341-345   -> afq_energy
//   timers                                  :50-77, 357 -> afq_stage_times
//
// Input: the in-memory data afqmc::Initialize leaves (initialize_serial.hpp:89-221) in
// the binary layout of synthetic.System.write_input, in place of the HDF5 file (no HDF5
// library is available to write one).  Differences from the reference's program, all
// additions: the time step comes from the input file (the reference fixes 0.01, :105);
// `-t no` parses its argument (the reference's getopt string gives `t` none, :120, so
// `-t no` dereferences a null optarg); the auxiliary fields come from the library's
// Philox4x32-10 stream keyed by -r instead of mt19937; -p, -e, -g, -d, -T, -P choose the
// numerical form, energy evaluation, graph substeps, device, Taylor order and printed
// digits; -b k combs the population after every k-th step (where the reference leaves
// branching out, :347); -c writes a checkpoint (walkers, W_data, Eshift, seed and step counters) after
// the last step and -R resumes from one: the fields are counter-based, so a resumed run
// repeats the uninterrupted one exactly (the reference has no checkpoint).  Errors print
// the library's message and exit with status 1.
#include <getopt.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <new>
#include <string>
#include <vector>

#include "afqmc_b200.h"

namespace {

struct Csr {
  int nrows = 0, ncols = 0;
  std::vector<int32_t> rowIndex, cols;
  std::vector<double> vals;   // interleaved complex
  long long nnz() const { return (long long)cols.size(); }
  afq_csr_z view() const {
    return afq_csr_z{nrows, ncols, rowIndex.data(), cols.data(), vals.data()};
  }
};

struct Input {
  int nmo = 0, naea = 0, naeb = 0, nchol = 0;
  double dt = 0.0;
  Csr Spvn, Vakbl;
  bool has_vakbl = false;
  std::vector<double> Propg1, haj, trial;   // interleaved complex
};

// Bounds-checked reader of the input file: every array size is checked against the
// bytes left before anything is allocated.
class Reader {
 public:
  explicit Reader(const std::string& path) : f_(path, std::ios::binary) {
    if (f_) {
      f_.seekg(0, std::ios::end);
      left_ = (long long)f_.tellg();
      f_.seekg(0, std::ios::beg);
    }
  }
  bool ok() const { return (bool)f_; }
  long long left() const { return left_; }
  template <class T>
  bool read(T* dst, long long count) {
    if (count < 0 || (long long)sizeof(T) * count > left_) return false;
    f_.read(reinterpret_cast<char*>(dst), (std::streamsize)(sizeof(T) * count));
    left_ -= (long long)sizeof(T) * count;
    return (bool)f_;
  }
  template <class T>
  bool vec(std::vector<T>& v, long long count) {
    if (count < 0 || (long long)sizeof(T) * count > left_) return false;
    v.resize((size_t)count);
    return read(v.data(), count);
  }

 private:
  std::ifstream f_;
  long long left_ = 0;
};

bool read_csr(Reader& r, Csr& m, int nrows, int ncols, const char* name, std::string* err) {
  int32_t dims[2];
  int64_t nnz = 0;
  if (!r.read(dims, 2) || !r.read(&nnz, 1)) {
    *err = std::string(name) + ": truncated header";
    return false;
  }
  if (dims[0] != nrows || dims[1] != ncols) {
    *err = std::string(name) + ": shape " + std::to_string(dims[0]) + " x " +
           std::to_string(dims[1]) + ", expected " + std::to_string(nrows) + " x " +
           std::to_string(ncols);
    return false;
  }
  if (nnz < 0 || nnz > 0x7fffffffLL) {
    *err = std::string(name) + ": bad nnz";
    return false;
  }
  m.nrows = nrows;
  m.ncols = ncols;
  if (!r.vec(m.rowIndex, (long long)nrows + 1) || !r.vec(m.cols, nnz) ||
      !r.vec(m.vals, 2 * nnz)) {
    *err = std::string(name) + ": truncated arrays";
    return false;
  }
  if (m.rowIndex[0] != 0 || m.rowIndex[nrows] != nnz) {
    *err = std::string(name) + ": rowIndex does not span the entries";
    return false;
  }
  return true;
}

bool read_input(const std::string& path, Input& in, std::string* err) {
  Reader r(path);
  if (!r.ok()) {
    *err = "cannot open " + path;
    return false;
  }
  char magic[8];
  if (!r.read(magic, 8) || std::memcmp(magic, "AFQINP01", 8) != 0) {
    *err = path + ": not a driver input file (magic AFQINP01)";
    return false;
  }
  int32_t dims[4];
  int32_t has_v = 0;
  if (!r.read(dims, 4) || !r.read(&in.dt, 1) || !r.read(&has_v, 1)) {
    *err = path + ": truncated header";
    return false;
  }
  in.nmo = dims[0];
  in.naea = dims[1];
  in.naeb = dims[2];
  in.nchol = dims[3];
  in.has_vakbl = has_v != 0;
  if (in.nmo <= 0 || in.naea <= 0 || in.nchol <= 0 || in.naea > in.nmo || !(in.dt > 0.0)) {
    *err = path + ": bad sizes in the header";
    return false;
  }
  if (in.naeb != in.naea) {   // initialize_serial.hpp:67-71
    *err = path + ": NAEA != NAEB (closed shell only)";
    return false;
  }
  const long long N = in.nmo, n = in.naea;
  if (!read_csr(r, in.Spvn, (int)(N * N), in.nchol, "Spvn", err)) return false;
  if (!r.vec(in.Propg1, 2 * N * N) || !r.vec(in.haj, 2 * 2 * n * N) ||
      !r.vec(in.trial, 2 * 2 * N * n)) {
    *err = path + ": truncated dense arrays";
    return false;
  }
  if (in.has_vakbl && !read_csr(r, in.Vakbl, (int)(2 * n * N), (int)(2 * n * N), "Vakbl", err))
    return false;
  if (r.left() != 0) {
    *err = path + ": " + std::to_string(r.left()) + " trailing bytes";
    return false;
  }
  return true;
}

// Checkpoint: everything a substep reads besides the Hamiltonian.  Little-endian binary:
//   char[8] "AFQCKP01"; int32 nmo, naea, nwalk, precision; int64 steps, step_tot;
//   uint64 seed; float64 eshift; float64 W[nwalk][2][nmo][naea] complex;
//   float64 W_data[nwalk][8] complex.
struct Checkpoint {
  int32_t nmo = 0, naea = 0, nwalk = 0, precision = 0;
  int64_t steps = 0, step_tot = 0;
  uint64_t seed = 0;
  double eshift = 0.0;
  std::vector<double> W, Wd;
};

bool write_checkpoint(const std::string& path, const Checkpoint& c, std::string* err) {
  std::ofstream f(path, std::ios::binary);
  auto put = [&](const void* p, size_t bytes) {
    f.write(static_cast<const char*>(p), (std::streamsize)bytes);
  };
  put("AFQCKP01", 8);
  const int32_t dims[4] = {c.nmo, c.naea, c.nwalk, c.precision};
  const int64_t steps[2] = {c.steps, c.step_tot};
  put(dims, sizeof dims);
  put(steps, sizeof steps);
  put(&c.seed, sizeof c.seed);
  put(&c.eshift, sizeof c.eshift);
  put(c.W.data(), sizeof(double) * c.W.size());
  put(c.Wd.data(), sizeof(double) * c.Wd.size());
  f.close();
  if (!f) *err = "cannot write " + path;
  return (bool)f;
}

bool read_checkpoint(const std::string& path, Checkpoint& c, std::string* err) {
  Reader r(path);
  if (!r.ok()) {
    *err = "cannot open " + path;
    return false;
  }
  char magic[8];
  int32_t dims[4];
  int64_t steps[2];
  if (!r.read(magic, 8) || std::memcmp(magic, "AFQCKP01", 8) != 0) {
    *err = path + ": not a checkpoint file (magic AFQCKP01)";
    return false;
  }
  if (!r.read(dims, 4) || !r.read(steps, 2) || !r.read(&c.seed, 1) || !r.read(&c.eshift, 1)) {
    *err = path + ": truncated header";
    return false;
  }
  c.nmo = dims[0];
  c.naea = dims[1];
  c.nwalk = dims[2];
  c.precision = dims[3];
  c.steps = steps[0];
  c.step_tot = steps[1];
  if (c.nmo <= 0 || c.naea <= 0 || c.nwalk <= 0 || c.steps < 0 || c.step_tot < 0) {
    *err = path + ": bad header";
    return false;
  }
  if (!r.vec(c.W, 4LL * c.nwalk * c.nmo * c.naea) || !r.vec(c.Wd, 16LL * c.nwalk) ||
      r.left() != 0) {
    *err = path + ": walker arrays do not match the header";
    return false;
  }
  return true;
}

void print_help() {
  std::printf("miniafqmc - QMCPACK AFQMC miniapp on the B200 library\n\n");
  std::printf("Options:\n");
  std::printf("-i                Number of MC steps (default: 10)\n");
  std::printf("-s                Number of substeps (default: 10)\n");
  std::printf("-w                Number of walkers (default: 16)\n");
  std::printf("-o                Number of substeps between orthogonalization (default: 10)\n");
  std::printf("-f                Input file name (default: ./afqmc.bin)\n");
  std::printf("-t                If set to no, do not use half-rotated transposed Cholesky "
              "matrix to calculate bias potential (default yes).\n");
  std::printf("-v                Verbose output\n");
  std::printf("-p                fp64 | mixed: numerical form (default fp64)\n");
  std::printf("-e                vakbl | chol | cv | cv2: local energy from the two-body "
              "matrix, the Cholesky factors, the learned control variate, or the two-level "
              "control variate (plain-bf16 exchange of every walker + learned residual; "
              "-p mixed) (default vakbl when the input has it, else chol)\n");
  std::printf("-g                Run each substep as one CUDA-graph launch (not with -t no)\n");
  std::printf("-d                CUDA device (default 0)\n");
  std::printf("-r                Seed of the auxiliary-field stream (default 11)\n");
  std::printf("-T                Taylor order of exp(vHS) (default 6)\n");
  std::printf("-P                Significant digits of the printed energies (default 6)\n");
  std::printf("-c                Write a checkpoint file after the last step\n");
  std::printf("-R                Resume from a checkpoint file (-i counts the steps before it)\n");
  std::printf("-b                Population control (comb) after every b-th step (default 0: "
              "none)\n");
}

struct Options {
  int nsteps = 10, nsubsteps = 10, nwalk = 16, northo = 10;
  std::string init_file = "afqmc.bin", checkpoint_out, resume_from;
  bool transposed = true, verbose = false, graph = false;
  int precision = AFQ_PREC_FP64;
  int energy = -1;   // -1: vakbl when present, else chol
  int cv_base = 0;   // -e cv2: the control variate's low-precision base
  int device = 0, taylor = 6, digits = 6, branch = 0;
  uint64_t seed = 11;
};

// parse; returns 0 to run, 1 after -h (the reference's exit status), 2 on a bad flag
int parse(int argc, char** argv, Options& o) {
  int opt;
  while ((opt = getopt(argc, argv, "hvgt:i:s:w:o:f:p:e:d:r:T:P:c:R:b:")) != -1) {
    switch (opt) {
      case 'h': print_help(); return 1;
      case 'i': o.nsteps = std::atoi(optarg); break;
      case 's': o.nsubsteps = std::atoi(optarg); break;
      case 'w': o.nwalk = std::atoi(optarg); break;
      case 'o': o.northo = std::atoi(optarg); break;
      case 't': o.transposed = std::string(optarg) != "no"; break;
      case 'f': o.init_file = optarg; break;
      case 'v': o.verbose = true; break;
      case 'g': o.graph = true; break;
      case 'p':
        if (!std::strcmp(optarg, "fp64")) o.precision = AFQ_PREC_FP64;
        else if (!std::strcmp(optarg, "mixed")) o.precision = AFQ_PREC_MIXED;
        else return 2;
        break;
      case 'e':
        if (!std::strcmp(optarg, "vakbl")) o.energy = AFQ_ENERGY_VAKBL;
        else if (!std::strcmp(optarg, "chol")) o.energy = AFQ_ENERGY_CHOLESKY;
        else if (!std::strcmp(optarg, "cv")) o.energy = AFQ_ENERGY_CV;
        else if (!std::strcmp(optarg, "cv2")) {
          o.energy = AFQ_ENERGY_CV;
          o.cv_base = 1;
        } else return 2;
        break;
      case 'd': o.device = std::atoi(optarg); break;
      case 'r': o.seed = std::strtoull(optarg, nullptr, 10); break;
      case 'T': o.taylor = std::atoi(optarg); break;
      case 'P': o.digits = std::atoi(optarg); break;
      case 'c': o.checkpoint_out = optarg; break;
      case 'R': o.resume_from = optarg; break;
      case 'b': o.branch = std::atoi(optarg); break;
      default: return 2;
    }
  }
  if (o.nsteps < 0 || o.nsubsteps < 0 || o.nwalk <= 0 || o.northo <= 0 || o.taylor < 0 ||
      o.digits <= 0 || o.digits > 17 || o.branch < 0)
    return 2;
  // the full-G path runs op by op (a graph substep is the transposed path)
  if (!o.transposed && o.graph) return 2;
  return 0;
}

// The library call's status, with its message; false after printing an error.
bool check(afq_status s, afq_handle* h, const char* what) {
  if (s == AFQ_OK) return true;
  std::cerr << " Error: " << what << ": " << afq_status_string(s);
  if (h) std::cerr << " (" << afq_last_error(h) << ")";
  std::cerr << std::endl;
  return false;
}

const char* kStageNames[AFQ_NSTAGES] = {
    "Mixed Density Matrix", "Bias Potential", "Sigma", "H-S Potential", "Propagation",
    "Overlap", "Other", "Orthgonalization", "Local Energy"};   // the reference's timer names

int run(const Options& o) {
  Input in;
  std::string err;
  std::cout << "***********************************************************\n";
  std::cout << "                 Initializing from input file              \n";
  std::cout << "***********************************************************\n";
  if (!read_input(o.init_file, in, &err)) {
    std::cerr << " Error initalizing data structures from input file: " << err << std::endl;
    return 1;
  }
  const int N = in.nmo, n = in.naea, nchol = in.nchol;
  const long long NAK = 2LL * n * N;
  Checkpoint resume;
  uint64_t seed = o.seed;
  if (!o.resume_from.empty()) {
    if (!read_checkpoint(o.resume_from, resume, &err)) {
      std::cerr << " Error: resume: " << err << std::endl;
      return 1;
    }
    if (resume.nmo != N || resume.naea != n || resume.nwalk != o.nwalk) {
      std::cerr << " Error: resume: the checkpoint holds " << resume.nwalk << " walkers of NMO "
                << resume.nmo << ", NAEA " << resume.naea << "; this run has " << o.nwalk
                << " of NMO " << N << ", NAEA " << n << std::endl;
      return 1;
    }
    seed = resume.seed;   // the fields continue the checkpointed stream
  }
  const int energy = o.energy >= 0 ? o.energy
                                   : (in.has_vakbl ? AFQ_ENERGY_VAKBL : AFQ_ENERGY_CHOLESKY);
  if (energy == AFQ_ENERGY_VAKBL && !in.has_vakbl) {
    std::cerr << " Error: -e vakbl needs the two-body matrix in the input file" << std::endl;
    return 1;
  }
  const bool need_lhalf = energy != AFQ_ENERGY_VAKBL;

  // half-rotation of the scaled Cholesky matrix (rotate.hpp:69-169) and, for the
  // Cholesky energies, the unscaled factors without the cutoff
  const afq_csr_z spvn = in.Spvn.view();
  Csr SpvnT;
  std::vector<double> Lhalf;
  {
    long long nnz = 0;
    if (need_lhalf) Lhalf.resize((size_t)2 * nchol * NAK);
    if (!check(afq_halfrotate(o.device, &spvn, N, n, nchol, in.trial.data(), 1e-6,
                              1.0 / std::sqrt(in.dt), &nnz, nullptr, nullptr, nullptr,
                              need_lhalf ? Lhalf.data() : nullptr),
               nullptr, "half-rotation"))
      return 1;
    SpvnT.nrows = nchol;
    SpvnT.ncols = (int)NAK;
    SpvnT.rowIndex.resize((size_t)nchol + 1);
    SpvnT.cols.resize((size_t)nnz);
    SpvnT.vals.resize((size_t)2 * nnz);
    long long nnz2 = 0;
    if (!check(afq_halfrotate(o.device, &spvn, N, n, nchol, in.trial.data(), 1e-6, 1.0, &nnz2,
                              SpvnT.rowIndex.data(), SpvnT.cols.data(), SpvnT.vals.data(),
                              nullptr),
               nullptr, "half-rotation") ||
        nnz2 != nnz) {
      if (nnz2 != nnz) std::cerr << " Error: half-rotation changed its entry count" << std::endl;
      return 1;
    }
  }

  std::cout << "\n";
  std::cout << "***********************************************************\n";
  std::cout << "                         Summary                           \n";
  std::cout << "***********************************************************\n";
  std::cout << "\n";
  std::cout << "  AFQMC system: \n"
            << "    NMO: " << N << "\n"
            << "    NAEA: " << in.naea << "\n"
            << "    NAEB: " << in.naeb << "\n"
            << "    dt: " << in.dt << "\n";
  std::cout << "\n";
  std::cout << "  Execution details: \n"
            << "    nsteps: " << o.nsteps << "\n"
            << "    nsubsteps: " << o.nsubsteps << "\n"
            << "    nwalk: " << o.nwalk << "\n"
            << "    northo: " << o.northo << "\n"
            << "    verbose: " << std::boolalpha << o.verbose << "\n"
            << "    # Chol Vectors: " << nchol << "\n"
            << "    transposed Spvn: " << o.transposed << "\n"
            << "    Chol. Matrix Sparsity: " << in.Spvn.nnz() / (double(nchol) * N * N) << "\n"
            << "    Hamiltonian Sparsity: "
            << (in.has_vakbl ? in.Vakbl.nnz() / (double(n) * n * N * N * 4.0) : 0.0) << "\n"
            << "    precision: " << (o.precision == AFQ_PREC_MIXED ? "mixed" : "fp64") << "\n"
            << "    energy: "
            << (energy == AFQ_ENERGY_VAKBL ? "vakbl"
                : energy == AFQ_ENERGY_CV   ? (o.cv_base ? "cv2" : "cv")
                                            : "chol")
            << "\n"
            << "    graph substeps: " << o.graph << "\n"
            << "    population control every: " << o.branch << " steps\n"
            << "    device: " << o.device << "\n"
            << "    seed: " << seed << std::endl;
  if (!o.resume_from.empty())
    std::cout << "    resumed after step " << resume.steps - 1 << " (substep " << resume.step_tot
              << ") from " << o.resume_from << std::endl;

  afq_system_desc desc{N, in.naea, in.naeb, nchol, o.nwalk, in.dt, o.taylor, o.precision,
                       o.device};
  afq_handle* h = nullptr;
  if (!check(afq_create(&desc, &h), nullptr, "afq_create")) return 1;
  struct Guard {
    afq_handle* h;
    ~Guard() { afq_destroy(h); }
  } guard{h};
  const afq_csr_z spvnT = SpvnT.view();
  const afq_csr_z vakbl = in.Vakbl.view();
  if (!check(afq_set_hamiltonian(h, &spvn, &spvnT, in.Propg1.data(), in.haj.data(),
                                 in.trial.data(), in.has_vakbl ? &vakbl : nullptr,
                                 need_lhalf ? Lhalf.data() : nullptr),
             h, "afq_set_hamiltonian"))
    return 1;
  Lhalf.clear();
  Lhalf.shrink_to_fit();
  if (energy == AFQ_ENERGY_CV &&
      !check(afq_cv_configure(h, 256, 1e-3, seed, 2000, 8), h, "afq_cv_configure"))
    return 1;
  if (energy == AFQ_ENERGY_CV && o.cv_base &&
      !check(afq_cv_set_base(h, 1), h, "afq_cv_set_base"))
    return 1;

  // walkers = conj(trial), weights 1 (miniafqmc_base.cpp:226-236)
  {
    std::vector<double> W((size_t)o.nwalk * 2 * N * n * 2), Wd((size_t)o.nwalk * 8 * 2, 0.0);
    const size_t per = (size_t)2 * N * n * 2;
    for (int w = 0; w < o.nwalk; w++) {
      for (size_t e = 0; e < per; e += 2) {
        W[w * per + e] = in.trial[e];
        W[w * per + e + 1] = -in.trial[e + 1];
      }
      Wd[(size_t)w * 16 + 2] = 1.0;   // W_data[w][1] = 1
    }
    const bool res = !o.resume_from.empty();
    if (!check(afq_set_walkers(h, res ? resume.W.data() : W.data(),
                               res ? resume.Wd.data() : Wd.data()),
               h, "afq_set_walkers") ||
        (res && !check(afq_set_eshift(h, resume.eshift), h, "afq_set_eshift")))
      return 1;
  }
  if (!o.graph && !check(afq_profile(h, 1), h, "afq_profile")) return 1;

  auto density_matrix = [&] {
    return o.transposed ? afq_mixed_density_matrix(h) : afq_mixed_density_matrix_full(h);
  };
  double Eav = 0.0;
  if (!check(afq_mixed_density_matrix(h), h, "mixed density matrix") ||
      !check(afq_energy(h, energy, &Eav), h, "energy"))
    return 1;
  std::cout << std::setprecision(o.digits);
  if (o.verbose) std::cout << "\n  initial energy: " << Eav << "\n";

  std::cout << "\n";
  std::cout << "***********************************************************\n";
  std::cout << "                     Beginning Steps                       \n";
  std::cout << "***********************************************************\n\n";
  std::cout << "# Step   Energy   \n";

  const auto t0 = std::chrono::steady_clock::now();
  int step = (int)resume.steps;
  uint64_t step_tot = (uint64_t)resume.step_tot;
  for (; step < o.nsteps; step++) {
    for (int sub = 0; sub < o.nsubsteps; sub++, step_tot++) {
      if (o.graph) {
        if (!check(afq_substep(h, seed, step_tot, o.northo), h, "substep")) return 1;
        continue;
      }
      // 1. density matrix and bias potential; 2. X and hybrid weight; 3. vHS;
      // 4. propagation; 5. overlaps; 6. weights and Eshift (miniafqmc_base.cpp:255-328)
      if (!check(density_matrix(), h, "mixed density matrix") ||
          !check(o.transposed ? afq_vbias(h) : afq_vbias_full(h), h, "vbias") ||
          !check(afq_sigma(h, seed, step_tot), h, "sigma") ||
          !check(afq_vhs(h), h, "vHS") || !check(afq_propagate(h), h, "propagate") ||
          !check(afq_overlaps(h, 1), h, "overlaps") ||
          !check(afq_update_weights(h), h, "weights"))
        return 1;
      if (step_tot > 0 && step_tot % (uint64_t)o.northo == 0) {   // miniafqmc_base.cpp:330-337
        if (!check(afq_orthogonalize(h), h, "orthogonalize") ||
            !check(afq_overlaps(h, 0), h, "overlaps"))
          return 1;
      }
    }
    if (!check(afq_mixed_density_matrix(h), h, "mixed density matrix") ||
        !check(afq_energy(h, energy, &Eav), h, "energy"))
      return 1;
    std::cout << step << "   " << Eav << "\n";
    // "Branching in real code would happen here" (miniafqmc_base.cpp:347)
    if (o.branch > 0 && (step + 1) % o.branch == 0 &&
        !check(afq_population_control(h, seed, step_tot), h, "population control"))
      return 1;
  }
  if (!check(afq_synchronize(h), h, "synchronize")) return 1;
  if (!o.checkpoint_out.empty()) {
    Checkpoint c;
    c.nmo = N;
    c.naea = n;
    c.nwalk = o.nwalk;
    c.precision = o.precision;
    c.steps = step;
    c.step_tot = (int64_t)step_tot;
    c.seed = seed;
    c.W.resize((size_t)4 * o.nwalk * N * n);
    c.Wd.resize((size_t)16 * o.nwalk);
    if (!check(afq_get_walkers(h, c.W.data(), c.Wd.data()), h, "afq_get_walkers") ||
        !check(afq_get_eshift(h, &c.eshift), h, "afq_get_eshift"))
      return 1;
    if (!write_checkpoint(o.checkpoint_out, c, &err)) {
      std::cerr << " Error: checkpoint: " << err << std::endl;
      return 1;
    }
  }
  const double total_s =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  std::cout << "\n";
  std::cout << "***********************************************************\n";
  std::cout << "                   Finished Calculation                    \n";
  std::cout << "***********************************************************\n\n";
  std::cout << std::setprecision(6);
  std::cout << "Timer                              GPU ms     kernels\n";
  std::cout << std::left << std::setw(32) << "Total (wall, ms)" << std::right << std::setw(10)
            << total_s * 1e3 << "\n";
  if (!o.graph) {
    double ms[AFQ_NSTAGES] = {};
    long long launches[AFQ_NSTAGES] = {};
    if (!check(afq_stage_times(h, ms, launches, 0), h, "stage times")) return 1;
    for (int s = 0; s < AFQ_NSTAGES; s++)
      std::cout << std::left << std::setw(32)
                << (s == AFQ_STAGE_DM && o.transposed ? "compact Mixed Density Matrix"
                                                      : kStageNames[s])
                << std::right << std::setw(10) << ms[s] << std::setw(12) << launches[s] << "\n";
  }
  {   // throughput of the timed loop (substeps and the per-step energies)
    const double ws = (double)o.nwalk * (double)(step_tot - (uint64_t)resume.step_tot);
    std::cout << "\n  walker-steps/s: " << (total_s > 0.0 ? ws / total_s : 0.0) << "  ("
              << (uint64_t)(step_tot - (uint64_t)resume.step_tot) << " substeps of "
              << o.nwalk << " walkers in " << total_s << " s)\n";
  }
  if (o.verbose) {
    double eshift = 0.0;
    if (check(afq_get_eshift(h, &eshift), h, "Eshift"))
      std::cout << "  final Eshift: " << std::setprecision(o.digits) << eshift << "\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  const int p = parse(argc, argv, o);
  if (p == 1) return 1;
  if (p == 2) {
    std::cerr << " Error: bad option (see -h)" << std::endl;
    return 1;
  }
  try {
    return run(o);
  } catch (const std::bad_alloc&) {
    std::cerr << " Error: out of host memory (input arrays or walkers too large)" << std::endl;
    return 1;
  }
}
