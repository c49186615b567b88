// ndyn_main.cpp -- directive-script driver over the C ABI: the host program
// that replaces Ndyn's Fortran main loop where no Fortran compiler exists.
//
//   ndyn_gpu [--mixed] [--fixed] [--device N] < input.sh
//
// Reads an Ndyn directive script on stdin from START (read_input,
// src/read_input.f90:2-219): Types, Pairs, Model (dump/xyz,
// src/read_input.f90:277-392), BoxSize, Skin, NeiMax, ReNeighbor,
// Isokinetic/Isoenergetic/Isobaric and their Aniso* forms, BoxVel /
// StopBoxVel, Velocity / Seed, OutFreq, StepNumber, ConfOutFreq, Print and
// Run, and prints the reference's write_thermo lines
// (src/read_input.f90:433-446) and writes its model files (write_model,
// src/read_input.f90:394-431).
// Every Run is one call of ndg_run (the dynamics prologue and loop,
// src/nd.f90:60-199) on the GPU.  --mixed selects NDG_PREC_MIXED, --fixed
// the corrected list semantics.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ndyn_gpu.h"

namespace {

std::vector<std::string> split(const std::string &line) {
  std::vector<std::string> w;
  size_t p = 0;
  while (p < line.size()) {
    while (p < line.size() && std::strchr(" \t\r\n", line[p])) ++p;
    if (p >= line.size()) break;
    size_t q = p;
    while (q < line.size() && !std::strchr(" \t\r\n", line[q])) ++q;
    w.push_back(line.substr(p, q - p));
    p = q;
  }
  return w;
}

std::string strip_comment(const std::string &s) {
  const size_t h = s.find('#');
  return h == std::string::npos ? s : s.substr(0, h);
}

// Fortran list-directed logical: optional '.', then T/t or F/f
bool parse_logical(const std::string &v) {
  size_t k = v.size() && v[0] == '.' ? 1 : 0;
  return k < v.size() && (v[k] == 'T' || v[k] == 't');
}

// Fortran G14.6 (write_thermo, src/read_input.f90:440)
std::string g14_6(double x) {
  char buf[64];
  if (x == 0.0) {
    std::snprintf(buf, sizeof buf, "%10s    ", std::signbit(x) ? "-0.00000" : "0.00000");
    return buf;
  }
  if (!std::isfinite(x)) {
    std::snprintf(buf, sizeof buf, "%14s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    return buf;
  }
  char e6[64];
  std::snprintf(e6, sizeof e6, "%.5e", x);
  const int ex = std::atoi(std::strchr(e6, 'e') + 1) + 1;  // x = 0.dddddd * 10^ex
  if (ex >= 0 && ex <= 6) {
    const int dec = 6 - ex;
    if (dec > 0) std::snprintf(buf, sizeof buf, "%10.*f    ", dec, x);
    else std::snprintf(buf, sizeof buf, "%9.0f.    ", x);  // F10.0 keeps the point
    return buf;
  }
  char tmp[64], dig[8];
  std::snprintf(tmp, sizeof tmp, "%.5e", std::fabs(x));
  dig[0] = tmp[0];
  std::memcpy(dig + 1, tmp + 2, 5);
  dig[6] = 0;
  char body[64];
  if (ex >= -99 && ex <= 99)
    std::snprintf(body, sizeof body, "%s0.%sE%c%02d", x < 0 ? "-" : "", dig, ex < 0 ? '-' : '+',
                  ex < 0 ? -ex : ex);
  else
    std::snprintf(body, sizeof body, "%s0.%s%c%03d", x < 0 ? "-" : "", dig, ex < 0 ? '-' : '+',
                  ex < 0 ? -ex : ex);
  std::snprintf(buf, sizeof buf, "%14s", body);
  return buf;
}

// Fortran ENw.d (engineering notation: a mantissa of 1 to 3 digits before
// the point, an exponent that is a multiple of 3), right-justified in w
std::string en_format(double x, int w, int d) {
  char body[64];
  if (x == 0.0 || !std::isfinite(x)) {
    if (x == 0.0) std::snprintf(body, sizeof body, "%s%.*fE+00", std::signbit(x) ? "-" : "", d, 0.0);
    else std::snprintf(body, sizeof body, "%s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
  } else {
    int e3 = 3 * (int)std::floor(std::floor(std::log10(std::fabs(x))) / 3.0);
    double m = x / std::pow(10.0, e3);
    char mant[48];
    std::snprintf(mant, sizeof mant, "%.*f", d, m);
    if (std::fabs(std::atof(mant)) >= 1000.0) {  // rounding carried into a fourth digit
      e3 += 3;
      m = x / std::pow(10.0, e3);
      std::snprintf(mant, sizeof mant, "%.*f", d, m);
    } else if (std::fabs(std::atof(mant)) < 1.0) {  // log10 landed just below a power of ten
      e3 -= 3;
      m = x / std::pow(10.0, e3);
      std::snprintf(mant, sizeof mant, "%.*f", d, m);
    }
    const int ae = e3 < 0 ? -e3 : e3;
    if (ae <= 99) std::snprintf(body, sizeof body, "%sE%c%02d", mant, e3 < 0 ? '-' : '+', ae);
    else std::snprintf(body, sizeof body, "%s%c%03d", mant, e3 < 0 ? '-' : '+', ae);
  }
  if ((int)std::strlen(body) > w) return std::string(w, '*');
  char out[64];
  std::snprintf(out, sizeof out, "%*s", w, body);
  return out;
}

void thermo_line(const ndg_thermo *t, void *) {
  std::printf(" %8d %s %s %s %s %s\n", t->step, g14_6(t->potential).c_str(),
              g14_6(t->kinetic).c_str(), g14_6(t->energy_error).c_str(),
              g14_6(t->pressure).c_str(), g14_6(t->volume).c_str());
  std::fflush(stdout);
}

// Seeded Maxwell-Boltzmann velocities with the reference's semantics
// (normalVelocityDistribution, src/nd.f90:1598-1621: sigma^2 = 2 kt /
// (3 m), mean removed).  The reference draws from gfortran's
// random_number; this driver uses SplitMix64 uniforms and the
// Kinderman-Monahan ratio-of-uniforms normal, the generator the CPU
// restatement uses, so both start from the same velocities.
uint64_t splitmix64(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

float uniform(uint64_t *st) {
  return ((float)(splitmix64(st) >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

float normal_ratio_of_uniforms(uint64_t *st) {
  const float s = 0.449871f, t = -0.386595f, a = 0.19600f, b = 0.25472f;
  const float r1 = 0.27597f, r2 = 0.27846f;
  for (;;) {
    const float u = uniform(st);
    float v = uniform(st);
    v = 1.7156f * (v - 0.5f);
    const float x = u - s, y = std::fabs(v) - t;
    const float q = x * x + y * (a * y - b * x);
    if (q < r1) return v / u;
    if (q > r2) continue;
    if (v * v < -4.0f * std::log(u) * u * u) return v / u;
  }
}

struct Driver {
  int precision = NDG_PREC_FP64, quirk = NDG_QUIRK_REF, device = 0;
  ndg_ctx *ctx = nullptr;
  int sys = -1;
  bool dirty = true;  // host state newer than the device's
  std::vector<std::string> tname;
  std::vector<double> mass, charge;
  // pair tables
  int npairs = 0, ptsize = 1000;
  double ptrmin = 0.25;
  std::vector<int> pairmat;
  std::vector<double> rcpair, ppair, fpair;
  // model
  std::vector<int> typ;
  std::vector<double> pos, vel, acc;
  double box[3] = {0, 0, 0};
  double boxset[3] = {10.0, 10.0, 10.0};
  std::string model, model_type = "xyz";
  uint64_t seed = 123456789ULL;
  ndg_control c{};
  // hold groups and their displacement conditions (src/read_input.f90:177-190)
  std::vector<int> hold;  // per atom: group, 0 = none
  std::vector<std::string> hname;
  std::vector<int> bcdir;
  std::vector<double> bcparm;
  bool holds_dirty = false;
  // spring pairs (their PairParams) and InitPos (src/read_input.f90:136,165)
  std::vector<int> spring;
  std::vector<double> pparams;
  bool springs_dirty = false, ipos_pending = false;
  std::vector<double> ipos;
  double ibox[3] = {0, 0, 0};
  // configuration output (ConfOutFreq [i] [type], src/read_input.f90:196-197)
  int conf_outs = 0;
  std::string model_out_type = "NA";

  // write_model, 'xyz' and 'dump' formats (src/read_input.f90:394-431); the
  // per-atom energy pene of the xyz records is zero (compute0 zeroes it,
  // src/nd.f90:251, and nothing adds to it)
  bool write_model(FILE *f, int step) const {
    const int np = (int)typ.size();
    if (model_out_type == "XYZ" || model_out_type == "xyz") {
      std::fprintf(f, "%8d\n\n", np);
      for (int i = 0; i < np; ++i) {
        const std::string &tn = tname.at(typ[i] - 1);
        std::fprintf(f, "%-4.4s ", tn.c_str());
        for (int k = 0; k < 3; ++k) std::fputs(en_format(pos[3 * (size_t)i + k], 14, 4).c_str(), f);
        for (int k = 0; k < 3; ++k) std::fputs(en_format(vel[3 * (size_t)i + k], 14, 4).c_str(), f);
        std::fputs(en_format(0.0, 14, 4).c_str(), f);
        std::fputc('\n', f);
      }
    } else if (model_out_type == "dump" || model_out_type == "trj") {
      std::fprintf(f, "ITEM: TIMESTEP\n%7d\nITEM: NUMBER OF ATOMS\n%7d\n", step, np);
      std::fprintf(f, "ITEM: BOX BOUNDS pp pp pp\n");
      for (int k = 0; k < 3; ++k) std::fprintf(f, "%12.4f%12.4f\n", 0.0, box[k]);
      std::fprintf(f, "ITEM: ATOMS id type xs ys zs\n");
      for (int i = 0; i < np; ++i) {
        // real(pos(1:3,i))+0.0: single precision, f9.5
        std::fprintf(f, "%7d %2d%9.5f%9.5f%9.5f\n", i + 1, typ[i], (double)(float)pos[3 * (size_t)i],
                     (double)(float)pos[3 * (size_t)i + 1], (double)(float)pos[3 * (size_t)i + 2]);
      }
    } else {
      std::fprintf(stderr, "ERROR: model out type: %s not supported\n", model_out_type.c_str());
      return false;
    }
    std::fflush(f);
    return true;
  }

  // positions as the device has them after a run (for domain selections)
  int sync_positions() {
    if (!ctx || sys < 0 || dirty) return NDG_OK;
    return ndg_get_state(ctx, sys, pos.data(), vel.data(), acc.data(), box);
  }

  int type_id(const std::string &t) const {
    for (size_t i = 0; i < tname.size(); ++i)
      if (tname[i] == t) return (int)i + 1;
    return 0;
  }

  // read_model, 'dump' and 'xyz' formats (src/read_input.f90:277-392)
  bool read_model() {
    FILE *f = std::fopen(model.c_str(), "r");
    if (!f) {
      std::fprintf(stderr, "read_model: ERROR: opening model file: %s\n", model.c_str());
      return false;
    }
    char line[1024];
    int np = 0;
    double b[3] = {boxset[0], boxset[1], boxset[2]};
    const bool dump = model_type == "dump" || model_type == "trj";
    auto next = [&]() { return std::fgets(line, sizeof line, f) != nullptr; };
    if (dump) {
      for (int k = 0; k < 3; ++k) next();
      next();
      np = std::atoi(line);
      next();
      for (int k = 0; k < 3; ++k) {
        float lm = 0, lx = 0;
        next();
        std::sscanf(line, "%f %f", &lm, &lx);
        b[k] = (double)(lx - lm);  // real(4) read, src/read_input.f90:334-336
      }
      next();
    } else {
      next();
      np = std::atoi(line);
      next();
    }
    typ.assign(np, 0);
    pos.assign(3 * (size_t)np, 0.0);
    for (int i = 0; i < np; ++i) {
      if (!next()) {
        std::fclose(f);
        return false;
      }
      if (dump) {
        int id = 0, ty = 0;
        float x[3] = {0, 0, 0};
        std::sscanf(line, "%d %d %f %f %f", &id, &ty, &x[0], &x[1], &x[2]);
        if (id < 1 || id > np) {
          std::fclose(f);
          return false;
        }
        typ[id - 1] = ty;
        for (int k = 0; k < 3; ++k) pos[3 * (size_t)(id - 1) + k] = (double)(x[k] - 0.5f);
      } else {
        char ct[64];
        double x[3] = {0, 0, 0};
        std::sscanf(line, "%63s %lf %lf %lf", ct, &x[0], &x[1], &x[2]);
        typ[i] = type_id(ct);
        if (!typ[i]) {
          std::fprintf(stderr, "ERROR: no atom type defined for atom %d\n", i + 1);
          std::fclose(f);
          return false;
        }
        for (int k = 0; k < 3; ++k) pos[3 * (size_t)i + k] = x[k] / b[k];
      }
    }
    std::fclose(f);
    for (int k = 0; k < 3; ++k) box[k] = b[k];
    vel.assign(3 * (size_t)np, 0.0);
    acc.assign(3 * (size_t)np, 0.0);  // the first Run starts from acc = 0
    dirty = true;
    std::printf("#  read_model: successfully read %8d model nodes.\n", np);
    return true;
  }

  // the device state back into the host copies (before a host-side change)
  bool pull() {
    if (sys < 0 || dirty) return true;
    return ndg_get_state(ctx, sys, pos.data(), vel.data(), acc.data(), box) == NDG_OK;
  }

  void velocity(float kt) {
    pull();
    const int np = (int)typ.size();
    uint64_t st = seed;
    double vt[3] = {0, 0, 0};
    for (int i = 0; i < np; ++i) {
      float nn[3];
      for (int d = 0; d < 3; ++d) nn[d] = normal_ratio_of_uniforms(&st);
      const float coeff = std::sqrt(2.0f * kt / (3.0f * (float)mass[typ[i] - 1]));
      for (int d = 0; d < 3; ++d) {
        vel[3 * (size_t)i + d] = (double)(nn[d] * coeff);
        vt[d] += vel[3 * (size_t)i + d];
      }
    }
    for (int d = 0; d < 3; ++d) vt[d] = vt[d] / (double)np;
    for (int i = 0; i < np; ++i)
      for (int d = 0; d < 3; ++d) vel[3 * (size_t)i + d] -= vt[d];
    dirty = true;
  }

  int run(int nsteps) {
    int rc = NDG_OK;
    if (!ctx) {
      rc = ndg_create(&ctx, device, precision);
      if (rc) return rc;
    }
    if (sys < 0) {
      rc = ndg_add_system(ctx, (int)typ.size(), (int)mass.size(), npairs, ptsize, ptrmin,
                          mass.data(), pairmat.data(), rcpair.data(), ppair.data(), fpair.data(),
                          typ.data(), pos.data(), vel.data(), acc.data(), box, &sys);
      if (rc) return rc;
    } else if (dirty) {
      rc = ndg_load_state(ctx, sys, pos.data(), vel.data(), acc.data(), box);
      if (rc) return rc;
    }
    dirty = false;
    c.quirk = quirk;
    rc = ndg_set_control(ctx, sys, &c);
    if (rc) return rc;
    if (springs_dirty) {
      bool any = false;
      for (int f : spring) any |= f != 0;
      rc = ndg_set_springs(ctx, sys, any ? spring.data() : nullptr, any ? pparams.data() : nullptr);
      if (rc) return rc;
      springs_dirty = false;
    }
    if (ipos_pending) {
      rc = ndg_set_initial_positions(ctx, sys, ipos.data(), ibox);
      if (rc) return rc;
      ipos_pending = false;
    }
    if (holds_dirty) {
      const bool any = !hname.empty();
      rc = ndg_set_holds(ctx, sys, any ? hold.data() : nullptr, (int)hname.size(),
                         any ? bcdir.data() : nullptr, any ? bcparm.data() : nullptr);
      if (rc) return rc;
      holds_dirty = false;
    }
    // dynamics (src/nd.f90:92-172): ConfOuts 0 means once per Run, 'NA'
    // means xyz (both persist); the model goes to out.<type> (appended) at
    // the start and wherever mod(step, ConfOuts) = 0.  The loop runs in
    // pieces that end there: ndg_run, then ndg_run_continue (one run).
    if (conf_outs == 0) conf_outs = nsteps;
    if (model_out_type == "NA") model_out_type = "xyz";
    FILE *mf = std::fopen(("out." + model_out_type).c_str(), "a");
    if (!mf) {
      std::fprintf(stderr, "dynamics: cannot open out.%s\n", model_out_type.c_str());
      return NDG_ERR_ARG;
    }
    if (!write_model(mf, c.step)) {
      std::fclose(mf);
      return NDG_ERR_ARG;
    }
    int done = 0;
    while (done < nsteps && rc == NDG_OK) {
      const int at = c.step + done;
      const int piece = std::min(nsteps - done, conf_outs - (((at % conf_outs) + conf_outs) % conf_outs));
      rc = done == 0 ? ndg_run(ctx, piece, thermo_line, nullptr)
                     : ndg_run_continue(ctx, piece, thermo_line, nullptr);
      done += piece;
      if (rc == NDG_OK && (c.step + done) % conf_outs == 0) {
        rc = ndg_get_state(ctx, sys, pos.data(), vel.data(), acc.data(), box);
        if (rc == NDG_OK && !write_model(mf, c.step + done)) rc = NDG_ERR_ARG;
      }
    }
    std::fclose(mf);
    if (rc) return rc;
    ndg_control after{};
    ndg_get_control(ctx, sys, &after);
    c.step = after.step;      // StepNumber carries over between Runs
    c.skin = after.skin;      // the default skin, once set, persists (src/nd.f90:77-79)
    c.neimax = after.neimax;  // so does the NeiMax estimate (src/nd.f90:84-88)
    return NDG_OK;
  }
};

}  // namespace

int main(int argc, char **argv) {
  Driver d;
  ndg_default_control(&d.c);
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--mixed")) d.precision = NDG_PREC_MIXED;
    else if (!std::strcmp(argv[a], "--fixed")) d.quirk = NDG_QUIRK_FIXED;
    else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) d.device = std::atoi(argv[++a]);
  }
  char raw[4096];
  bool started = false;
  while (std::fgets(raw, sizeof raw, stdin)) {
    auto w = split(raw);
    if (!w.empty() && w[0] == "START") {
      started = true;
      break;
    }
  }
  if (!started) {
    std::fprintf(stderr, "read_input: no START line\n");
    return 1;
  }
  int ln = 0;
  auto arg = [](const std::vector<std::string> &w, size_t n) -> std::string {
    return n < w.size() ? w[n] : std::string("0");
  };
  while (std::fgets(raw, sizeof raw, stdin)) {
    ++ln;
    auto w = split(strip_comment(raw));
    if (w.empty()) continue;
    const std::string &k = w[0];
    if (k == "ConfOutFreq") {
      d.conf_outs = std::atoi(arg(w, 1).c_str());
      if (w.size() >= 3) d.model_out_type = w[2];
    } else if (k == "help" || k == "WritePotentialTable") {
      // no output on the timestep path
    } else if (k == "BoxSize") {
      for (int q = 0; q < 3; ++q) d.boxset[q] = std::atof(arg(w, q + 1).c_str());
    } else if (k == "Model") {
      d.model = arg(w, 1);
      if (w.size() >= 3) d.model_type = w[2];
      if (!d.read_model()) return 2;
      // a new model holds no atoms (read_model, src/read_input.f90:294-296)
      d.hold.assign(d.typ.size(), 0);
      d.hname.clear();
      d.bcdir.clear();
      d.bcparm.clear();
      d.holds_dirty = true;
    } else if (k == "Seed") {
      d.seed = std::strtoull(arg(w, 1).c_str(), nullptr, 10);
    } else if (k == "Velocity") {
      d.velocity((float)std::atof(arg(w, 1).c_str()));
    } else if (k == "ReNeibour" || k == "ReNeighbor") {
      d.c.renei = parse_logical(arg(w, 1));
      if (w.size() >= 3) d.c.renei_freq = std::atoi(w[2].c_str());
    } else if (k == "Skin") {
      d.c.skin = std::atof(arg(w, 1).c_str());
    } else if (k == "NeiMax") {
      d.c.neimax = std::atoi(arg(w, 1).c_str());
    } else if (k == "Types") {
      const int nt = std::atoi(arg(w, 1).c_str());
      d.tname.clear();
      d.mass.clear();
      d.charge.clear();
      for (int i = 0; i < nt; ++i) {
        if (!std::fgets(raw, sizeof raw, stdin)) return 3;
        auto tw = split(raw);
        d.tname.push_back(tw.size() > 0 ? tw[0].substr(0, 8) : "");
        d.mass.push_back(tw.size() > 1 ? std::atof(tw[1].c_str()) : 0.0);
        d.charge.push_back(tw.size() > 2 ? std::atof(tw[2].c_str()) : 0.0);
      }
    } else if (k == "Pairs") {
      const int np = std::atoi(arg(w, 1).c_str());
      d.ptrmin = w.size() >= 3 ? std::atof(w[2].c_str()) : 0.25;
      d.ptsize = w.size() >= 4 ? std::atoi(w[3].c_str()) : 1000;
      const int nt = (int)d.mass.size();
      std::vector<char> names(8 * (size_t)np, ' ');
      std::vector<double> par(4 * (size_t)np, 0.0), q(np, 0.0);
      d.pairmat.assign((size_t)nt * nt, 0);
      for (int i = 0; i < np; ++i) {
        if (!std::fgets(raw, sizeof raw, stdin)) return 3;
        auto tw = split(strip_comment(raw));
        const int a = tw.size() > 0 ? d.type_id(tw[0]) : 0;
        const int b = tw.size() > 1 ? d.type_id(tw[1]) : 0;
        const bool sym = tw.size() > 2 && tw[2] == "sym";
        if (tw.size() > 3) std::memcpy(names.data() + 8 * i, tw[3].c_str(), std::min<size_t>(8, tw[3].size()));
        for (size_t j = 4; j < tw.size() && j < 8; ++j) par[4 * i + (j - 4)] = std::atof(tw[j].c_str());
        if (!a || !b) {
          std::fprintf(stderr, "Pairs: unknown type on pair %d\n", i + 1);
          return 4;
        }
        q[i] = d.charge[a - 1] * d.charge[b - 1];
        // PairMat(a,b) (column-major), the reverse order too for 'sym'; an
        // 'asym' pair acts one way and selects compute1 (src/read_input.f90:125-133)
        d.pairmat[(a - 1) + (size_t)(b - 1) * nt] = i + 1;
        if (sym) d.pairmat[(b - 1) + (size_t)(a - 1) * nt] = i + 1;
      }
      d.npairs = np;
      d.spring.assign(np, 0);
      d.pparams = par;
      for (int i = 0; i < np; ++i) {
        // PairParams(1,:) defaults to the global rcut where a line gives none
        // (src/read_input.f90:123); a spring's rc, D0, sc, Vol follow
        d.spring[i] = std::strncmp(names.data() + 8 * i, "spring  ", 8) == 0;
      }
      d.springs_dirty = true;
      d.ppair.assign((size_t)(d.ptsize + 1) * np, 0.0);
      d.fpair.assign((size_t)(d.ptsize + 1) * np, 0.0);
      std::vector<double> rc2(np), dr2(np);
      const int rc = ndg_build_pair_tables(np, d.ptsize, d.ptrmin, names.data(), par.data(),
                                           q.data(), d.ppair.data(), d.fpair.data(), rc2.data(),
                                           dr2.data());
      if (rc) {
        std::fprintf(stderr, "Pairs: %s\n", ndg_error_string(rc));
        return 4;
      }
      d.rcpair.assign(np, 0.0);
      double rcut = 0.0;
      for (int i = 0; i < np; ++i) {
        d.rcpair[i] = par[4 * i];
        rcut = std::max(rcut, par[4 * i]);
      }
      std::printf("# Global maximum cutoff radius: %g\n", rcut);
    } else if (k == "Isokinetic") {
      d.c.isokinetic = 1;
      d.c.ke_target = std::atof(arg(w, 1).c_str());
      d.c.ke_parm = std::atof(arg(w, 2).c_str());
      if (w.size() >= 4) d.c.ke_freq = std::atoi(w[3].c_str());
    } else if (k == "Anisokinetic") {
      d.c.isokinetic = 0;
    } else if (k == "Isoenergetic") {
      d.c.isoenergetic = 1;
      d.c.e_parm = std::atof(arg(w, 1).c_str());
      if (w.size() >= 3) d.c.e_freq = std::atoi(w[2].c_str());
    } else if (k == "Anisoenergetic") {
      d.c.isoenergetic = 0;
    } else if (k == "Isobaric") {
      d.c.isobaric = 1;
      for (int q = 0; q < 3; ++q) d.c.p_target[q] = std::atof(arg(w, q + 1).c_str());
      d.c.p_parm = std::atof(arg(w, 4).c_str());
      if (w.size() >= 6) d.c.p_freq = std::atoi(w[5].c_str());
    } else if (k == "Anisobaric") {
      d.c.isobaric = 0;
    } else if (k == "BoxVel") {
      d.c.box_load = 1;
      for (int q = 0; q < 3; ++q) d.c.box_vel[q] = std::atof(arg(w, q + 1).c_str());
    } else if (k == "StopBoxVel") {
      d.c.box_load = 0;
    } else if (k == "Exec") {
      std::printf("# Exec not executed\n");
    } else if (k == "Print") {
      const std::string s(raw);
      std::printf("# %s", s.size() > 6 ? s.c_str() + 6 : "\n");
    } else if (k == "OutFreq") {
      d.c.out_steps = std::atoi(arg(w, 1).c_str());
    } else if (k == "StepNumber") {
      d.c.step = std::atoi(arg(w, 1).c_str());
    } else if (k == "Hold") {
      // Hold NAME typ ID | Hold NAME dom rec INSIDE xmin xmax ymin ymax zmin zmax
      // (setGroup 'h', src/nd.f90:1625-1700; rectangular domains,
      // src/domtype.f90:299-343, compared in FP32 on fractional positions)
      if (d.typ.empty()) {
        std::fprintf(stderr, "Hold: no model\n");
        return 4;
      }
      d.hold.resize(d.typ.size(), 0);
      d.hname.push_back(arg(w, 1));
      d.bcdir.insert(d.bcdir.end(), 3, 0);
      d.bcparm.insert(d.bcparm.end(), 3, 0.0);
      const int g = (int)d.hname.size();
      const std::string how = arg(w, 2).substr(0, 3);
      if (how == "typ") {
        const int t = std::atoi(arg(w, 3).c_str());
        for (size_t i = 0; i < d.typ.size(); ++i)
          if (d.typ[i] == t) d.hold[i] = g;
      } else if (how == "dom" && arg(w, 3) == "rec" && w.size() >= 11) {
        const std::string ins = arg(w, 4);
        const bool inside = !(ins == "F" || ins == "f" || ins == ".false." || ins == "false");
        float lo[3], hi[3];
        int dir[3];
        for (int a = 0; a < 3; ++a) {
          lo[a] = (float)std::atof(w[5 + 2 * a].c_str());
          hi[a] = (float)std::atof(w[6 + 2 * a].c_str());
          dir[a] = (std::fabs(hi[a]) + std::fabs(lo[a])) < 1.17549435e-38f ? 0 : 1;
        }
        if (d.sync_positions()) return 4;
        for (size_t i = 0; i < d.typ.size(); ++i) {
          bool in = true;
          for (int a = 0; a < 3; ++a) {
            const float x = (float)d.pos[3 * i + a];
            if (dir[a] && !(x > lo[a] && x <= hi[a])) in = false;
          }
          if (in == inside) d.hold[i] = g;
        }
      } else {
        std::fprintf(stderr, "Hold: only 'typ ID' and 'dom rec ...' selections are supported\n");
        return 4;
      }
      d.holds_dirty = true;
    } else if (k == "Disp") {
      // Disp NAME dx dy dz: per axis a displacement per step (fractional), F = free
      int g = 0;
      for (size_t q = 0; q < d.hname.size(); ++q)
        if (d.hname[q] == arg(w, 1)) g = (int)q + 1;
      if (!g) {
        std::fprintf(stderr, "Disp: unknown hold group %s\n", arg(w, 1).c_str());
        return 4;
      }
      for (int a = 0; a < 3; ++a) {
        const std::string v = arg(w, 2 + a);
        const bool on = !v.empty() && v != "F";
        d.bcdir[3 * (g - 1) + a] = on;
        d.bcparm[3 * (g - 1) + a] = on ? std::atof(v.c_str()) : 0.0;
      }
      d.holds_dirty = true;
    } else if (k == "InitPos") {
      // initPositionSet, only with spring pairs (src/read_input.f90:165)
      bool any = false;
      for (int f : d.spring) any |= f != 0;
      if (!any) {
        std::printf("# WARNING: InitPos not applicable without a spring potential\n");
      } else {
        if (d.sync_positions()) return 4;
        d.ipos = d.pos;
        for (int a = 0; a < 3; ++a) d.ibox[a] = d.box[a];
        d.ipos_pending = true;
      }
    } else if (k == "ClearHolds") {
      d.hold.assign(d.typ.size(), 0);
      d.hname.clear();
      d.bcdir.clear();
      d.bcparm.clear();
      d.holds_dirty = true;
    } else if (k == "HoldBufferSize") {
      // group storage grows as needed
    } else if (k == "Run") {
      const int nsteps = std::atoi(arg(w, 1).c_str());
      if (w.size() >= 3) d.c.dt = std::atof(w[2].c_str());
      if (d.typ.empty() || !d.npairs) {
        std::fprintf(stderr, "Run: no model or no pairs\n");
        return 5;
      }
      std::printf("#  Step   Potential     Kinetic        EnergyError    pressure       volume\n");
      const int rc = d.run(nsteps);
      if (rc) {
        std::fprintf(stderr, "dynamics: %s (%d) %s\n", ndg_error_string(rc), rc,
                     ndg_last_error(d.ctx));
        return 5;
      }
      int nup = 0;
      ndg_get_list_updates(d.ctx, d.sys, &nup);
      std::printf("# Number of neighbour list updates:%8d\n", nup);
      std::fflush(stdout);
    } else if (k == "END" || k == "DONE" || k == "end" || k == "done") {
      break;
    } else if (k == "EXIT" || k == "exit" || k == "quit" || k == "abort") {
      break;
    } else {
      std::fprintf(stderr, "#  read_input: unsupported directive: %s line:%4d\n", k.c_str(), ln);
    }
  }
  if (d.ctx) ndg_destroy(d.ctx);
  return 0;
}
