// marfa_cli.cpp -- the `marfa` command: the reference's main program
// (app/main.f90) driving libmarfa_gpu.so through its C ABI.
//
//   marfa Molecule StartWV EndWV DatabaseSlug CutOff TargetValue AtmProfileFile
//         [precision fp64|fp32c] [chi none|tonkov|pollack|perrin] [device]
//
// Same positional arguments, input paths (data/databases/<slug>.<NN>,
// data/Atmospheres/<file>, data/TIPS/TIPS.dat relative to the working
// directory), output directory (output/ptTables/<Molecule>_<start>-<end>_<timestamp>),
// info.txt, latest_run.txt and PT-table files ('1__.ptbin' ...; record
// int((start+1)/10), 81,924 bytes) as the reference (EnvironmentSetup.f90:34-166,
// main.f90:81-180).  Exit codes are the reference's `stop` codes; arguments
// beyond the seventh are optional, the reference ignores them.
#include <sys/stat.h>
#include <sys/types.h>
#include <fcntl.h>
#include <unistd.h>

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "marfa_gpu.h"

namespace {

int species_code(const std::string &m) {
  static const char *names[] = {"H2O", "CO2", "O3", "N2O", "CO", "CH4", "O2", "NO", "SO2", "NO2", "NH3", "HNO3"};
  for (int i = 0; i < 12; ++i)
    if (m == names[i]) return i + 1;
  return 0;
}

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// list-directed numbers: blanks and commas separate values
std::vector<double> numbers(const std::string &line) {
  std::vector<double> v;
  std::string t = line;
  for (char &c : t)
    if (c == ',') c = ' ';
  std::istringstream is(t);
  std::string tok;
  while (is >> tok) {
    char *end = nullptr;
    const double x = std::strtod(tok.c_str(), &end);
    if (end == tok.c_str() || *end) return {};
    v.push_back(x);
  }
  return v;
}

void usage(int argc) {
  std::printf(" Insufficient number of arguments.\n");
  std::printf(" Expected at least 7 arguments, but received %d\n", argc);
  std::printf(" Usage: marfa Molecule StartWV EndWV DatabaseSlug CutOff TargetValue AtmProfileFile\n");
  std::printf("        [precision fp64|fp32c] [chi none|tonkov|pollack|perrin] [device]\n");
}

} // namespace

int main(int argc, char **argv) {
  const int nargs = argc - 1;
  if (nargs < 7) {
    usage(nargs);
    return 1;
  }
  const std::string molecule = trim(argv[1]);
  const std::string start_txt = trim(argv[2]), end_txt = trim(argv[3]);
  const std::string slug = trim(argv[4]), cut_txt = trim(argv[5]);
  const std::string target = trim(argv[6]), profile_file = trim(argv[7]);
  // FP64 is the drop-in arithmetic; fp32c is the faster form, opted into
  const std::string precision = nargs >= 8 ? trim(argv[8]) : "fp64";
  const std::string chi_name = nargs >= 9 ? trim(argv[9]) : "none";
  const int device = nargs >= 10 ? std::atoi(argv[10]) : 0;
  char *e1 = nullptr, *e2 = nullptr, *e3 = nullptr;
  const double start_wv = std::strtod(start_txt.c_str(), &e1);
  const double end_wv = std::strtod(end_txt.c_str(), &e2);
  const double cutoff = std::strtod(cut_txt.c_str(), &e3);
  if (*e1 || *e2 || *e3) {
    std::printf(" Error: StartWV, EndWV and CutOff must be numbers\n");
    return 1;
  }
  if (target != "ACS" && target != "VAC") {
    std::printf(" Error: Invalid targetValue \"%s\". Must be either \"ACS\" (Absorption cross-section) or "
                "\"VAC\" (Volume absorption coefficient).\n", target.c_str());
    return 2;
  }
  int chi = -1;
  const char *chis[] = {"none", "tonkov", "pollack", "perrin"};
  for (int i = 0; i < 4; ++i)
    if (chi_name == chis[i]) chi = i;
  if (chi < 0 || (precision != "fp32c" && precision != "fp64")) {
    std::printf(" Error: precision must be fp32c or fp64 and chi one of none, tonkov, pollack, perrin\n");
    return 1;
  }

  // atmospheric profile (Atmsosphere.f90:29-60)
  const std::string prof_path = "data/Atmospheres/" + profile_file;
  std::ifstream pf(prof_path);
  if (!pf) {
    std::printf(" Error: cannot open %s\n", prof_path.c_str());
    return 7;
  }
  std::string line;
  std::getline(pf, line); // title (A20), ignored
  std::getline(pf, line);
  std::vector<double> head = numbers(line);
  if (head.empty()) {
    std::printf(" Error: Unable to read data from file \"%s\".\n", prof_path.c_str());
    return 7;
  }
  const int levels = (int)head[0];
  if (levels > 200) {
    std::printf("WARNING: input number of atmospheric levels is bigger than 200\n");
    return 6;
  }
  std::vector<double> P(levels), T(levels), n(levels);
  for (int l = 0; l < levels; ++l) {
    std::vector<double> row;
    if (std::getline(pf, line)) row = numbers(line);
    if (row.size() < 4) {
      std::printf(" Error: Unable to read data from file \"%s\".\n Check the data format in the atmospheric file\n",
                  prof_path.c_str());
      return 7;
    }
    P[l] = row[1];
    T[l] = row[2];
    n[l] = row[3];
  }

  // TIPS (EnvironmentSetup.f90:169-184)
  std::ifstream tf("data/TIPS/TIPS.dat");
  if (!tf) {
    std::printf(" Error: cannot open data/TIPS/TIPS.dat\n");
    return 9;
  }
  std::getline(tf, line);
  std::vector<double> th = numbers(line);
  if (th.size() < 2) return 9;
  const int n_iso = (int)th[0], n_temp = (int)th[1];
  std::vector<double> tips((size_t)n_iso * n_temp);
  std::vector<double> all;
  while ((int)all.size() < n_iso * n_temp && std::getline(tf, line)) {
    std::vector<double> v = numbers(line);
    all.insert(all.end(), v.begin(), v.end());
  }
  if ((int)all.size() < n_iso * n_temp) {
    std::printf(" Error: short TIPS table\n");
    return 9;
  }
  std::copy(all.begin(), all.begin() + (size_t)n_iso * n_temp, tips.begin());

  // molecule and database (main.f90:68-74, 196-212)
  const int code = species_code(molecule);
  if (code == 0) {
    std::printf(" ERROR: unsupported molecule: %s\n", molecule.c_str());
    return 8;
  }
  char ext[8];
  std::snprintf(ext, sizeof ext, "%02d", code);
  const std::string db_path = "data/databases/" + slug + "." + ext;
  std::ifstream df(db_path, std::ios::binary | std::ios::ate);
  if (!df) {
    std::printf(" ERROR: when reading file with spectral data.\n");
    return 9;
  }
  const std::streamsize db_bytes = df.tellg();
  df.seekg(0);
  std::vector<marfa_line_record> lines((size_t)db_bytes / sizeof(marfa_line_record));
  df.read((char *)lines.data(), (std::streamsize)(lines.size() * sizeof(marfa_line_record)));

  // output directory, info.txt, latest_run.txt (EnvironmentSetup.f90:98-166)
  std::time_t now = std::time(nullptr);
  std::tm tmv = *std::localtime(&now);
  char stamp[32];
  std::strftime(stamp, sizeof stamp, "%Y%m%d_%H%M%S", &tmv);
  const std::string sub = molecule + "_" + std::to_string((long long)start_wv) + "-" +
                          std::to_string((long long)end_wv) + "_" + stamp;
  const std::string parent = "output/ptTables/";
  const std::string dir = parent + sub;
  if (mkdir(dir.c_str(), 0755) != 0) {
    std::printf(" Error: Failed to create directory %s\n", dir.c_str());
    return 3;
  }
  std::printf(" Directory for storing PT-tables is created: %s\n", dir.c_str());
  {
    FILE *f = std::fopen((dir + "/info.txt").c_str(), "w");
    if (!f) {
      std::printf(" Error: Unable to create info file at %s/info.txt\n", dir.c_str());
      return 4;
    }
    std::fprintf(f, "Command-Line Arguments:\nInput Molecule: %s\nStart Wavenumber: %s\nEnd Wavenumber: %s\n"
                    "Cut Off: %s\nTarget Value: %s\nAtmospheric Profile File: %s\n",
                 molecule.c_str(), start_txt.c_str(), end_txt.c_str(), cut_txt.c_str(), target.c_str(),
                 profile_file.c_str());
    std::fclose(f);
    std::printf(" Info file created at: %s/info.txt\n", dir.c_str());
    FILE *g = std::fopen((parent + "latest_run.txt").c_str(), "w");
    if (!g) {
      std::printf(" Error: Unable to create latest run file at %slatest_run.txt\n", parent.c_str());
      return 5;
    }
    std::fprintf(g, "%s\n", sub.c_str());
    std::fclose(g);
  }

  marfa_ctx *ctx = nullptr;
  int rc = marfa_ctx_create(lines.data(), (int64_t)lines.size(), tips.data(), n_iso, n_temp, device, &ctx);
  if (rc) {
    std::printf(" ERROR: device setup failed (status %d)\n", rc);
    return rc < 256 ? rc : 1;
  }
  marfa_run run;
  run.start_wv = start_wv;
  run.end_wv = end_wv;
  run.cutoff = cutoff;
  run.target = target == "VAC" ? MARFA_TARGET_VAC : MARFA_TARGET_ACS;
  run.mol_code = code;
  run.chi = chi;
  run.shape = MARFA_SHAPE_VOIGT;
  run.precision = precision == "fp64" ? MARFA_PREC_FP64 : MARFA_PREC_FP32C;
  const int nsub = marfa_num_subintervals(start_wv, end_wv);
  std::vector<int> recno(nsub);
  for (int i = 0; i < nsub; ++i) recno[i] = marfa_record_number(start_wv, i);

  // levels in chunks: one library call per chunk, then one file per level
  const size_t rec_floats = MARFA_NT, rec_bytes = rec_floats * 4;
  const int chunk = std::max(1, (int)std::min<size_t>(levels, ((size_t)2 << 30) / (nsub * rec_bytes + 1)));
  std::vector<float> out((size_t)chunk * nsub * rec_floats);
  for (int l0 = 0; l0 < levels; l0 += chunk) {
    const int nl = std::min(chunk, levels - l0);
    rc = marfa_compute(ctx, &run, P.data() + l0, T.data() + l0, n.data() + l0, nl, out.data(), nullptr);
    if (rc) {
      std::printf(" ERROR: %s (status %d)\n", marfa_last_error(ctx), rc);
      marfa_ctx_destroy(ctx);
      return rc < 256 ? rc : 1;
    }
    for (int l = 0; l < nl; ++l) {
      const int lev = l0 + l + 1;
      char label[8];
      std::snprintf(label, sizeof label, "%d", lev);
      std::string name(label);
      name.append(3 - name.size(), '_');
      const std::string path = dir + "/" + name + ".ptbin";
      const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
      if (fd < 0) {
        std::printf(" ERROR: cannot write %s\n", path.c_str());
        marfa_ctx_destroy(ctx);
        return 4;
      }
      for (int s = 0; s < nsub; ++s) {
        const float *rec = out.data() + ((size_t)l * nsub + s) * rec_floats;
        const off_t off = (off_t)(recno[s] - 1) * (off_t)rec_bytes;
        if (pwrite(fd, rec, rec_bytes, off) != (ssize_t)rec_bytes) {
          std::printf(" ERROR: short write to %s\n", path.c_str());
          close(fd);
          marfa_ctx_destroy(ctx);
          return 4;
        }
      }
      close(fd);
      std::printf(" %d  of  %d  atmospheric levels is being processed ...\n", lev, levels);
    }
  }
  marfa_ctx_destroy(ctx);
  std::printf("  *** Congratulations! PT-tables have been calculated! ***\n");
  return 0;
}
