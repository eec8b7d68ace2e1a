// ASCII seismogram writer with the reference's file naming and format
// (src/io/seismogram/writer.cpp:23-88): one "time value" line per sample,
// both in std::scientific, files NET.STA.S2.BX{X,Z}.sem{d,v,a},
// NET.STA.S2.PRE.semp and, for SH, NET.STA.S2.BXY.sem{d,v,a}.
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <stdexcept>
#include <string>
#include <vector>

#include "problem.hpp"

namespace sfb {

void write_seismograms_ascii(const Problem &P, const float *seis, int ntypes, int nrec, int max_sig,
                             const std::string &dir) {
  static const char *ext[] = {"semd", "semv", "sema", "semp", "semr"};
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);  // the folder may not exist yet
  for (int r = 0; r < nrec; ++r) {
    const Receiver &rc = P.receivers[r];
    for (int it = 0; it < ntypes; ++it) {
      const int type = P.seismogram_types[it];
      std::vector<std::string> names;
      const std::string stem = dir + "/" + rc.network + "." + rc.station + ".S2.";
      if (type == SEIS_PRESSURE) {
        if (P.elastic_sh) throw std::runtime_error("Pressure seismograms are not supported for SH waves");
        names = {stem + "PRE." + ext[type]};
      } else if (P.elastic_sh) {
        names = {stem + "BXY." + ext[type]};
      } else {
        names = {stem + "BXX." + ext[type], stem + "BXZ." + ext[type]};
      }
      for (size_t c = 0; c < names.size(); ++c) {
        std::ofstream f(names[c]);
        if (!f) throw std::runtime_error("Could not open seismogram file: " + names[c]);
        for (int isig = 0; isig < max_sig; ++isig) {
          const double t = static_cast<double>(static_cast<float>(
              isig * static_cast<float>(P.dt) * P.nstep_between_samples + static_cast<float>(P.t0)));
          const float v = seis[((static_cast<size_t>(isig) * ntypes + it) * nrec + r) * 2 + c];
          f << std::scientific << t << " " << std::scientific << v << "\n";
        }
      }
    }
  }
}

}  // namespace sfb
