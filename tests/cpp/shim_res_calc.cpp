// A res_calc driver written against the reference's host API, compiled
// against include/fot_problem.hpp (the engine's drop-in) instead of the
// reference's problem.hpp.  It reads the reference's text inputs from a
// directory (res_calc.cu:10-40), optionally reorders and partitions, runs the
// hierarchical or global loop and writes the un-permuted result.
//
//   shim_res_calc <dir> <iterations> <exec: hier|global> <reorder: 0|1> <out>
//
// Built with -DSHIM_SOA=1 it runs Problem<true> (component-major point data);
// the text files are point-major in both layouts, as the reference's readers.
#include <fstream>
#include <iostream>
#include <string>

#include "fot_problem.hpp"

using fot::compat::Problem;

#ifndef SHIM_SOA
#define SHIM_SOA 0
#endif

int main(int argc, char **argv) {
  if (argc < 6) return 2;
  const std::string dir = argv[1];
  const unsigned num = std::stoul(argv[2]);
  const std::string exec = argv[3];
  const bool reorder = std::string(argv[4]) == "1";
  try {
    std::ifstream mesh_res(dir + "/mesh_res"), mesh_x(dir + "/mesh_x"), mesh_q(dir + "/mesh_q"),
        mesh_adt(dir + "/mesh_adt");
    Problem<SHIM_SOA != 0> problem({&mesh_res, &mesh_x, &mesh_q, &mesh_adt}, {2, 2, 2, 2},
                           {{4, sizeof(double)}, {2, sizeof(double)}, {4, sizeof(double)},
                            {1, sizeof(double)}},
                           {}, 128);
    std::ifstream data_res(dir + "/data_res"), data_x(dir + "/data_x"), data_q(dir + "/data_q"),
        data_adt(dir + "/data_adt");
    problem.readPointData<double>(data_res, 0);
    problem.readPointData<double>(data_x, 1);
    problem.readPointData<double>(data_q, 2);
    problem.readPointData<double>(data_adt, 3);
    if (reorder) {
      problem.reorder();
      problem.partition(1.001f);
      problem.reorderToPartition();
      problem.renumberPoints();
    }
    if (exec == "hier")
      problem.loopGPUHierarchical<fot::compat::res_calc::StepGPUHierarchical>(num);
    else
      problem.loopGPUCellCentred<fot::compat::res_calc::StepGPUGlobal>(num);
    std::ofstream out(argv[5]);
    out.precision(17);
    problem.writePointData<double>(out);
  } catch (const fot::compat::Error &e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  } catch (const fot::compat::InvalidInputFile &e) {
    std::cerr << "invalid input " << e.input_type << " line " << e.line << "\n";
    return 1;
  }
  return 0;
}
