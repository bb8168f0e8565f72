// Test harness for the drop-in check: the reference's unmodified
// sol/rcwa_bridge.cpp, compiled against this engine's RCWASolver/Layer
// headers, driven by the globals that sol/input_data.c would set.  Reads the
// RCWA keys of an .ofd file (rcwa, rcwalayer, rcwadispersion, rcwaincidence,
// planewave, frequency1, title; the meanings of sol/input_data.c:400-520) and
// calls rcwa_run(), which writes rcwa_efficiency.csv and rcwa_orders.csv.
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref by oracle/build_ref.sh).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "orcwa_rcwa.h"
#include "rcwa_hdf5.h"

extern "C" {
int NRcwaHarmonics = 0, NRcwaHarmonicsY = 0, NRcwaLayer = 0, NRcwaPole = 0, IRcwaIncidence = 0;
double RcwaPeriod = 0, RcwaPeriodY = 0, RcwaTheta = 0, RcwaPhi = 0;
rcwalayer_t* RcwaLayer = nullptr;
rcwapole_t* RcwaPole = nullptr;
int NFreq1 = 0;
double* Freq1 = nullptr;
char Title[256] = "";
void monitor1(FILE* fp, const char s[]) {
  if (fp) std::fprintf(fp, "%s\n", s);
}
int rcwa_run(FILE* fp_log);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s file.ofd\n", argv[0]);
    return 2;
  }
  std::ifstream in(argv[1]);
  std::string line;
  std::vector<rcwalayer_t> layers;
  std::vector<rcwapole_t> poles;
  bool have_period_y = false;
  double pw_theta = 0, pw_phi = 0;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    std::string key, eq;
    ss >> key >> eq;
    if (eq != "=") continue;
    std::vector<std::string> t;
    std::string w;
    while (ss >> w) t.push_back(w);
    if (key == "title") {
      std::strncpy(Title, line.c_str() + line.find('=') + 2, sizeof(Title) - 1);
    } else if (key == "rcwa" && (t.size() == 2 || t.size() == 4)) {
      NRcwaHarmonics = std::atoi(t[0].c_str());
      RcwaPeriod = std::atof(t[1].c_str());
      if (t.size() == 4) {
        NRcwaHarmonicsY = std::atoi(t[2].c_str());
        RcwaPeriodY = std::atof(t[3].c_str());
        have_period_y = true;
      }
    } else if (key == "rcwalayer" && t.size() >= 4) {
      rcwalayer_t l{};
      l.eps1 = std::atof(t[0].c_str());
      l.eps2 = std::atof(t[1].c_str());
      l.fill = std::atof(t[2].c_str());
      l.thickness = std::atof(t[3].c_str());
      l.eps1i = t.size() >= 6 ? std::atof(t[4].c_str()) : 0.0;
      l.eps2i = t.size() >= 6 ? std::atof(t[5].c_str()) : 0.0;
      l.fill_y = t.size() >= 7 ? std::atof(t[6].c_str()) : 1.0;
      layers.push_back(l);
    } else if (key == "rcwadispersion" && t.size() == 6) {
      rcwapole_t p{};
      p.layer = std::atoi(t[0].c_str()) - 1;
      p.side = std::atoi(t[1].c_str());
      p.einf = std::atof(t[2].c_str());
      p.ae = std::atof(t[3].c_str());
      p.be = std::atof(t[4].c_str());
      p.ce = std::atof(t[5].c_str());
      poles.push_back(p);
    } else if (key == "rcwaincidence" && t.size() == 2) {
      IRcwaIncidence = 1;
      RcwaTheta = std::atof(t[0].c_str());
      RcwaPhi = std::atof(t[1].c_str());
    } else if (key == "planewave" && t.size() >= 2) {
      pw_theta = std::atof(t[0].c_str());
      pw_phi = std::atof(t[1].c_str());
    } else if (key == "frequency1" && t.size() >= 3) {
      const double f0 = std::atof(t[0].c_str()), f1 = std::atof(t[1].c_str());
      const int div = std::atoi(t[2].c_str());
      NFreq1 = div + 1;
      Freq1 = (double*)std::malloc(sizeof(double) * NFreq1);
      for (int n = 0; n < NFreq1; ++n) Freq1[n] = f0 + n * (div > 0 ? (f1 - f0) / div : 0.0);
    }
  }
  if (!have_period_y) RcwaPeriodY = RcwaPeriod;
  if (!IRcwaIncidence) {
    RcwaTheta = pw_theta;
    RcwaPhi = pw_phi;
  }
  NRcwaLayer = (int)layers.size();
  RcwaLayer = layers.data();
  NRcwaPole = (int)poles.size();
  RcwaPole = poles.empty() ? nullptr : poles.data();
  const int rc = rcwa_run(stdout);
  std::free(Freq1);
  return rc;
}
