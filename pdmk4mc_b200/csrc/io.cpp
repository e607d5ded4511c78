// Particle files: the reference's read_particle_info (src/utils.cpp:14-28).
// The first line is a header and is skipped; every further line that starts
// with four numbers x y z q gives one particle (anything after the fourth
// number is ignored); lines that do not are skipped.
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace pdmk {

// false when the file cannot be opened
bool read_particle_info(const std::string& filename, std::vector<double>& xyzq) {
  std::ifstream in(filename);
  if (!in) return false;
  xyzq.clear();
  std::string line;
  std::getline(in, line);  // header
  while (std::getline(in, line)) {
    std::istringstream is(line);
    double x, y, z, q;
    if (!(is >> x >> y >> z >> q)) continue;
    xyzq.insert(xyzq.end(), {x, y, z, q});
  }
  return true;
}

}  // namespace pdmk
