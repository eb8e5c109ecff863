// Known-answer driver in the shape of the reference's test programs
// (src/test-ldc-stru-nelem10.cpp:22-62):
//   test-ldc-stru <mesh prefix> <control file> <solver-options file> <reference result>
// Exit code 0 and "Result matches" when StabFEM::checkResult accepts.
#include <cstdio>
#include <string>

#include "StabFEM.h"

int main(int argc, char *argv[])
{
  if (argc < 5) {
    fprintf(stderr, "usage: %s <mesh prefix> <control> <options> <reference result>\n", argv[0]);
    return 2;
  }
  std::string meshfile = argv[1], controlfile = argv[2], optionsfile = argv[3], resultfile = argv[4];
  StabFEM stabfem;
  stabfem.verbose = false;
  stabfem.readSolverOptions(optionsfile);
  stabfem.readInputData(meshfile);
  stabfem.readControlParameters(controlfile);
  stabfem.prepareInputData();
  if (stabfem.setSolver(1, nullptr, false) != 0) return 1;
  if (stabfem.solveFullyImplicit() != 0) return 1;
  printf(" Simulation is completed. ... Checking the solution... \n ");
  if (stabfem.checkResult(resultfile) != 0) {
    printf("\n\n\n Result does not match \n\n\n");
    return 1;
  }
  printf("\n\n\n Result matches \n\n\n");
  printf("\n\n\n Test is successful \n\n\n ");
  return 0;
}
