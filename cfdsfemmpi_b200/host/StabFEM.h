// StabFEM -- C++ host driver over the cfdgpu C ABI.
//
// Keeps the public interface of the reference's driver class
// (src/base/StabFEM.h:89-153) and its three input formats, so the
// reference's main program and test drivers keep their shape; the PETSc
// solver object and the element loop are replaced by one cfdgpu_step call per
// time step (src/base/StabFEM2.cpp:632-799).
#pragma once

#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "cfdgpu.h"

class StabFEM {
 public:
  int ndim = 0, ndof = 0, npElem = 0;
  int nNode_global = 0, nElem_global = 0, nDBC = 0, nFBC = 0, nOutputFaceLoads = 0;
  int stepsMax = 0, outputFreq = 1, tis = 0, fileCount = 0;
  double conv_tol = 0.0, rhoInf = 0.0, timeFinal = 0.0, dt = 0.0;
  double elemData[50] = {0}, timeData[50] = {0};
  double computerTimeAssembly = 0, computerTimeSolver = 0, computerTimePostprocess = 0, computerTimePattern = 0,
         computerTimeTimeLoop = 0;

  std::vector<std::vector<double>> node_coords;
  std::vector<std::vector<int>> elemConn;
  std::vector<std::vector<double>> DirichletBCs;   // node (0-based), dof (0-based), value
  std::vector<int> outputNodes;
  std::vector<double> soln;                        // host copy of SolutionData::soln
  std::map<std::string, std::string> options;      // PETSc-style options
  std::string infilename;
  bool writeVTU = false;
  bool verbose = true;

  cfdgpu_handle *gpu = nullptr;

  StabFEM() = default;
  ~StabFEM();

  int deallocatePetscObjects();
  void readInputData(std::string &fname);
  void readControlParameters(std::string &fname);
  void readSolverOptions(const std::string &fname);
  void prepareInputData();
  int setSolver(int slv, int *parm = nullptr, bool cIO = false);
  int solveFullyImplicit();
  void postProcess();
  int writeResult(std::string &fname);
  int checkResult(std::string &fname);
  int printComputerTimes();
  std::string solverDescription() const;

 private:
  std::ofstream fout_convdata;
  cfdgpu_solver_opts opts_{};
};
