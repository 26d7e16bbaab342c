/* ORACLE — TEST INFRASTRUCTURE ONLY.  Runs the reference's own INI reader and
   problem setups (inputData, file_access.cpp:61-270, compiled unmodified) on
   a deck and writes the initial state it builds, so that the device problem
   generators can be compared with it bit for bit.

     ref_setup deck.ini out.bin

   out.bin: int32 nx, ny; float64 dx, dy, gamma; int32 bc[4] (left, right,
   bottom, top, BoundaryCondition values); then the U[0][0] block, 8 x
   (nx+4) x (ny+4) float64.  inputData also writes the deck's binary hint
   file into the working directory. */
#include <cstdio>
#include <cstdlib>
#include <string>

#include "mhd2d.hpp"

/* The reference program defines this in main.cpp (main.cpp:365-396). */
void criticalError(ReturnStatus error, const std::string message) {
  std::fprintf(stderr, "Critical error (%d): %s\n", int(error), message.c_str());
  std::exit(3);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s deck.ini out.bin\n", argv[0]);
    return 2;
  }
  t_output og, ong;
  t_params params;
  t_data data;
  inputData(argv[1], og, ong, params, data);
  FILE* f = std::fopen(argv[2], "wb");
  if (!f) return 4;
  const int n[2] = {params.nx, params.ny};
  const double d[3] = {params.dx, params.dy, params.gamma};
  const int bc[4] = {int(params.boundary[params.b_left]), int(params.boundary[params.b_right]),
                     int(params.boundary[params.b_bottom]), int(params.boundary[params.b_top])};
  std::fwrite(n, sizeof n, 1, f);
  std::fwrite(d, sizeof d, 1, f);
  std::fwrite(bc, sizeof bc, 1, f);
  const size_t tot = size_t(PRB_DIM) * (params.nx + 4) * (params.ny + 4);
  std::fwrite(data.U[0][0], sizeof(double), tot, f);
  std::fclose(f);
  return 0;
}
