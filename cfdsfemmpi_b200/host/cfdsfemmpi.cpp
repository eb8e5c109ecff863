// Main program with the reference's command line (src/cfdsfemmpi.cpp:22-89):
//   cfdsfemmpi <mesh prefix> <control file> <solver-options file>
#include <cstdio>
#include <string>

#include "StabFEM.h"

int main(int argc, char *argv[])
{
  if (argc < 4) {
    fprintf(stderr, " Error in input data \n You must enter name of input file\n Aborting...\n");
    return 1;
  }
  std::string meshfile = argv[1], controlfile = argv[2], optionsfile = argv[3];
  printf("\n    Input mesh file         = %s \n ", meshfile.c_str());
  printf("\n    Control parameters file = %s \n ", controlfile.c_str());
  printf("\n    PETSc options file      = %s \n ", optionsfile.c_str());
  StabFEM stabfem;
  stabfem.readSolverOptions(optionsfile);
  stabfem.readInputData(meshfile);
  stabfem.readControlParameters(controlfile);
  stabfem.prepareInputData();
  if (stabfem.setSolver(1, nullptr, false) != 0) return 1;
  printf("\n Solver: %s\n", stabfem.solverDescription().c_str());
  if (stabfem.solveFullyImplicit() != 0) return 1;
  stabfem.printComputerTimes();
  printf("\n\n\n Program is successful \n\n\n ");
  stabfem.deallocatePetscObjects();
  return 0;
}
