// spray_driver.cpp -- a C++ host program driving the B200 spray update through
// pmp::SprayParticleContainer (the C++ mirror of the reference's container),
// the way PeleLMeX's time step drives SprayParticleContainer: per step one
// moveKickDrift (sub-cycled, moving) and one moveKick, sources zeroed before
// each call and accumulated by the caller.
//
// Input/output is a directory of raw files (written and read by
// pelemp_b200/problem_io.py):
//   meta.txt            "nspec N", "species A B C", "nfuel F", "nboxes B",
//                       "steps S", "flow_dt X", "state_ghosts G",
//                       "source_ghosts G", "spray_cfl_lev C"
//   inputs.bin comps.bin geom.bin     the pmp_spray_inputs / pmp_spray_comps /
//                                      pmp_geometry structs, raw bytes
//   boxes.bin                          nboxes pmp_box
//   state_views.bin source_views.bin   nboxes pmp_box_view (p ignored)
//   state_<b>.bin                      the state fab of box b (float64)
//   pos_<b>.bin rdata_<b>.bin id_<b>.bin  droplets of box b (SoA)
// Outputs: out_pos_<b>.bin out_rdata_<b>.bin out_id_<b>.bin, out_src_<b>.bin
// (the sum of the deposits of every call).
//
// Usage: pmp_spray_driver <dir> [device]
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "SprayParticleContainer.H"

namespace {

template <class T>
std::vector<T> read_raw(const std::string& path)
{
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    throw std::runtime_error("cannot read " + path);
  }
  const std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<T> v(static_cast<size_t>(n) / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), n);
  return v;
}

template <class T>
void write_raw(const std::string& path, const T* p, size_t n)
{
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n * sizeof(T)));
}

template <class T>
T read_struct(const std::string& path)
{
  auto v = read_raw<unsigned char>(path);
  T t;
  if (v.size() != sizeof(T)) {
    throw std::runtime_error("size mismatch in " + path);
  }
  std::memcpy(&t, v.data(), sizeof(T));
  return t;
}

size_t extent(const pmp_box_view& v)
{
  const long long nx = v.hi[0] - v.lo[0] + 1;
  const long long ny = v.hi[1] - v.lo[1] + 1;
  const long long nz = v.hi[2] - v.lo[2] + 1;
  return static_cast<size_t>((v.ncomp - 1) * v.nstride + (nz - 1) * v.kstride + (ny - 1) * v.jstride + nx);
}

}  // namespace

int main(int argc, char** argv)
{
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <problem dir> [device]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int device = argc > 2 ? std::atoi(argv[2]) : 0;
  try {
    std::ifstream meta(dir + "/meta.txt");
    std::string line;
    std::vector<std::string> species;
    int nfuel = 0, nboxes = 0, steps = 0, state_ghosts = 0, source_ghosts = 0;
    double flow_dt = 0., cfl = 0.;
    while (std::getline(meta, line)) {
      std::istringstream is(line);
      std::string key;
      is >> key;
      if (key == "species") {
        std::string s;
        while (is >> s) {
          species.push_back(s);
        }
      } else if (key == "nfuel") {
        is >> nfuel;
      } else if (key == "nboxes") {
        is >> nboxes;
      } else if (key == "steps") {
        is >> steps;
      } else if (key == "flow_dt") {
        is >> flow_dt;
      } else if (key == "state_ghosts") {
        is >> state_ghosts;
      } else if (key == "source_ghosts") {
        is >> source_ghosts;
      } else if (key == "spray_cfl_lev") {
        is >> cfl;
      }
    }
    pmp::SprayParticleContainer spc(species, nfuel, device);
    spc.setViewsOnHost(true);  // the fabs below are host arrays
    spc.readSprayParams(read_struct<pmp_spray_inputs>(dir + "/inputs.bin"));
    spc.AssignSprayComps(read_struct<pmp_spray_comps>(dir + "/comps.bin"));
    spc.setGeometry(read_struct<pmp_geometry>(dir + "/geom.bin"));
    auto boxes = read_raw<pmp_box>(dir + "/boxes.bin");
    spc.setGrids(boxes);
    const int nr = PMP_PSTATE_NUM(nfuel);
    std::vector<std::vector<double>> pos(nboxes), rdata(nboxes);
    std::vector<std::vector<int>> ids(nboxes);
    for (int b = 0; b < nboxes; ++b) {
      const std::string s = std::to_string(b);
      pos[b] = read_raw<double>(dir + "/pos_" + s + ".bin");
      rdata[b] = read_raw<double>(dir + "/rdata_" + s + ".bin");
      ids[b] = read_raw<int>(dir + "/id_" + s + ".bin");
      const long long n = static_cast<long long>(ids[b].size());
      pmp_particles p{};
      p.layout = PMP_LAYOUT_SOA;
      p.where = PMP_WHERE_HOST;
      p.n = n;
      for (int d = 0; d < 3; ++d) {
        p.pos[d] = pos[b].data() + d * n;
      }
      for (int r = 0; r < nr; ++r) {
        p.rdata[r] = rdata[b].data() + r * n;
      }
      p.id = ids[b].data();
      spc.setParticles(b, p);
    }
    auto st_views = read_raw<pmp_box_view>(dir + "/state_views.bin");
    auto sr_views = read_raw<pmp_box_view>(dir + "/source_views.bin");
    std::vector<std::vector<double>> state(nboxes), src(nboxes), total(nboxes);
    for (int b = 0; b < nboxes; ++b) {
      state[b] = read_raw<double>(dir + "/state_" + std::to_string(b) + ".bin");
      if (state[b].size() < extent(st_views[b])) {
        throw std::runtime_error("state file smaller than its view");
      }
      st_views[b].p = state[b].data();
      src[b].assign(extent(sr_views[b]), 0.0);
      total[b].assign(extent(sr_views[b]), 0.0);
      sr_views[b].p = src[b].data();
    }
    long long substeps = 0;
    for (int step = 0; step < steps; ++step) {
      for (int do_move = 1; do_move >= 0; --do_move) {
        for (auto& s : src) {
          std::fill(s.begin(), s.end(), 0.0);
        }
        if (do_move) {
          spc.moveKickDrift(st_views, sr_views, 0, flow_dt, 0.0, false, false, state_ghosts,
                            source_ghosts, true, nullptr, cfl);
        } else {
          spc.moveKick(st_views, sr_views, 0, flow_dt, 0.0, false, false, state_ghosts,
                       source_ghosts, nullptr, cfl);
        }
        // the host sources are read next: wait for the call (device errors
        // surface here)
        spc.synchronize();
        substeps += spc.stats().substeps;
        for (int b = 0; b < nboxes; ++b) {
          for (size_t i = 0; i < src[b].size(); ++i) {
            total[b][i] += src[b][i];
          }
        }
      }
    }
    for (int b = 0; b < nboxes; ++b) {
      const std::string s = std::to_string(b);
      const long long n = static_cast<long long>(ids[b].size());
      pmp_particles p{};
      p.layout = PMP_LAYOUT_SOA;
      p.where = PMP_WHERE_HOST;
      p.n = n;
      for (int d = 0; d < 3; ++d) {
        p.pos[d] = pos[b].data() + d * n;
      }
      for (int r = 0; r < nr; ++r) {
        p.rdata[r] = rdata[b].data() + r * n;
      }
      p.id = ids[b].data();
      spc.getParticles(b, p);
      write_raw(dir + "/out_pos_" + s + ".bin", pos[b].data(), pos[b].size());
      write_raw(dir + "/out_rdata_" + s + ".bin", rdata[b].data(), rdata[b].size());
      write_raw(dir + "/out_id_" + s + ".bin", ids[b].data(), ids[b].size());
      write_raw(dir + "/out_src_" + s + ".bin", total[b].data(), total[b].size());
    }
    std::printf("pmp_spray_driver: ok substeps=%lld\n", substeps);
    return 0;
  } catch (const pmp::SprayAbort& e) {
    std::fprintf(stderr, "pmp_spray_driver: abort (%d, box %d, droplet %lld): %s\n", e.code(),
                 e.info().box, e.info().particle, e.what());
    return 10 + e.code();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pmp_spray_driver: %s\n", e.what());
    return 1;
  }
}
