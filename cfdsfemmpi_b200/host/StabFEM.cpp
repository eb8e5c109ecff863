// StabFEM -- C++ host driver over the cfdgpu C ABI (see StabFEM.h).
#include "StabFEM.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>

namespace {
double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

StabFEM::~StabFEM() { deallocatePetscObjects(); }

int StabFEM::deallocatePetscObjects()
{
  if (gpu) cfdgpu_destroy(gpu);
  gpu = nullptr;
  return 0;
}

// Mesh file: StabFEM::readInputData (src/base/StabFEM.cpp:80-264)
void StabFEM::readInputData(std::string &fname)
{
  infilename = fname;
  std::ifstream infile(infilename + ".dat");
  if (infile.fail()) {
    std::cerr << "\n\n Could not open the input nodes file \n\n";
    exit(1);
  }
  std::string s, v[3];
  infile >> s >> ndim >> s >> npElem >> s >> nNode_global >> s >> nElem_global >> s >> nDBC >> s >> nFBC >> s >>
      nOutputFaceLoads;
  ndof = ndim + 1;
  node_coords.assign(nNode_global, std::vector<double>(ndim));
  infile >> s;
  double tmp;
  for (int i = 0; i < nNode_global; i++) {
    infile >> tmp;
    for (int c = 0; c < ndim; c++) infile >> node_coords[i][c];
  }
  infile >> s;
  if (npElem != 3 && npElem != 4 && npElem != 8) {
    std::cerr << " Invalid npElem " << npElem << std::endl;
    exit(-1);
  }
  elemConn.assign(nElem_global, std::vector<int>(npElem));
  int a[12];
  for (int e = 0; e < nElem_global; e++) {
    for (int k = 0; k < 4 + npElem; k++) infile >> a[k];
    for (int k = 0; k < npElem; k++) elemConn[e][k] = a[4 + k] - 1;
  }
  infile >> v[0] >> v[1] >> v[2];
  DirichletBCs.clear();
  for (int k = 0; k < nDBC; k++) {
    int n1, n2;
    double val;
    infile >> n1 >> n2 >> val;
    DirichletBCs.push_back({double(n1 - 1), double(n2 - 1), val});
  }
  infile >> s;
  outputNodes.resize(nOutputFaceLoads);
  for (int k = 0; k < nOutputFaceLoads; k++) {
    infile >> outputNodes[k];
    outputNodes[k] -= 1;
  }
  fout_convdata.open(infilename + "-forces.dat", std::ios::out | std::ios::trunc);
  if (fout_convdata.fail()) {
    std::cout << " Could not open the output file for writing forces " << std::endl;
    exit(1);
  }
  fout_convdata.setf(std::ios::fixed);
  fout_convdata.setf(std::ios::showpoint);
  fout_convdata.precision(14);
}

// Control file: positional, keywords ignored (src/base/StabFEM.cpp:268-322)
void StabFEM::readControlParameters(std::string &fname)
{
  std::ifstream infile(fname);
  if (infile.fail()) {
    std::cout << " Could not open 'control-parameters.dat' file " << std::endl;
    exit(-1);
  }
  timeData[1] = 1.0;
  timeData[2] = 0.0;
  std::string s;
  infile >> s >> elemData[0] >> s >> elemData[1] >> s >> elemData[2] >> elemData[3] >> elemData[4] >> s >>
      elemData[8] >> elemData[9] >> elemData[10] >> s >> tis >> s >> rhoInf >> s >> dt >> s >> timeFinal >> s >>
      stepsMax >> s >> outputFreq >> s >> conv_tol;
}

// PETSc options file (passed to PetscInitialize in the reference, src/cfdsfemmpi.cpp:40)
void StabFEM::readSolverOptions(const std::string &fname)
{
  std::ifstream in(fname);
  std::string line;
  while (std::getline(in, line)) {
    auto hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    std::istringstream ls(line);
    std::string k, v;
    if (!(ls >> k) || k[0] != '-') continue;
    std::string rest;
    while (ls >> v) rest += (rest.empty() ? "" : " ") + v;
    options[k] = rest;
  }
}

void StabFEM::prepareInputData()
{
  if (!((ndim == 2 && (npElem == 3 || npElem == 4)) || (ndim == 3 && (npElem == 4 || npElem == 8)))) {
    std::cerr << " Invalid npElem " << npElem << std::endl;
    exit(-1);
  }
  soln.assign((size_t)nNode_global * ndof, 0.0);
}

std::string StabFEM::solverDescription() const
{
  const char *pc[] = {"none", "jacobi", "pbjacobi", "bjacobi"};
  std::ostringstream o;
  if (opts_.ksp_type == CFDGPU_KSP_BCGS) o << "BCGS";
  else if (opts_.ksp_type == CFDGPU_KSP_PREONLY) o << "preonly";
  else o << "GMRES(" << opts_.restart << ")";
  o << " pc=" << pc[opts_.pc_type];
  if (opts_.pc_type == CFDGPU_PC_BJACOBI_ILU) {
    o << "[" << (opts_.bjacobi_blocks > 0 ? opts_.bjacobi_blocks : 1) << " x ";
    if (opts_.ilu_levels < 0) o << "LU]";
    else o << "ILU(" << opts_.ilu_levels << ")]";
  }
  o << " rtol=" << opts_.rtol << " max_it=" << opts_.max_it;
  return o.str();
}

// setSolver + prepareMatrixPattern (src/base/StabFEM2.cpp:10-319).  PETSc
// option names with PETSc's defaults for a serial run; a method the library
// does not implement is an error, never replaced by another one.
int StabFEM::setSolver(int slv, int *parm, bool cIO)
{
  (void)slv; (void)parm; (void)cIO;
  auto get = [&](const char *k, const char *d) {
    auto it = options.find(k);
    return it == options.end() ? std::string(d) : it->second;
  };
  const std::string ksp = get("-ksp_type", "gmres"), pc = get("-pc_type", "ilu");
  opts_ = cfdgpu_solver_opts{};
  opts_.restart = 30; opts_.rtol = 1e-5; opts_.atol = 1e-50; opts_.dtol = 1e4; opts_.max_it = 10000;
  opts_.precision = CFDGPU_PREC_FP64; opts_.inner_restart = 0;
  opts_.inner_rtol = 1e-2; opts_.inner_restart = 20; opts_.reuse_tangent = 1; opts_.refine_rtol = 1e-10;
  opts_.newton_rtol = 0.0;
  if (ksp == "gmres") opts_.ksp_type = CFDGPU_KSP_GMRES;
  else if (ksp == "bcgs") opts_.ksp_type = CFDGPU_KSP_BCGS;
  else if (ksp == "preonly") opts_.ksp_type = CFDGPU_KSP_PREONLY;
  else {
    std::cerr << " -ksp_type " << ksp << " is not implemented (gmres, bcgs, preonly)" << std::endl;
    return CFDGPU_EINVAL;
  }
  opts_.bjacobi_blocks = 1;
  if (pc == "none") opts_.pc_type = CFDGPU_PC_NONE;
  else if (pc == "jacobi") opts_.pc_type = CFDGPU_PC_JACOBI;
  else if (pc == "pbjacobi") opts_.pc_type = CFDGPU_PC_PBJACOBI;
  else if (pc == "ilu" || pc == "lu") {
    opts_.pc_type = CFDGPU_PC_BJACOBI_ILU;
    opts_.ilu_levels = (pc == "lu") ? -1 : std::atoi(get("-pc_factor_levels", "0").c_str());
  } else if (pc == "bjacobi") {
    const std::string sub = get("-sub_pc_type", "ilu");
    if (sub != "ilu" && sub != "lu") {
      std::cerr << " -sub_pc_type " << sub << " is not implemented (ilu, lu)" << std::endl;
      return CFDGPU_EINVAL;
    }
    if (get("-sub_ksp_type", "preonly") != "preonly") {
      std::cerr << " -sub_ksp_type must be preonly" << std::endl;
      return CFDGPU_EINVAL;
    }
    opts_.pc_type = CFDGPU_PC_BJACOBI_ILU;
    opts_.ilu_levels = (sub == "lu") ? -1 : std::atoi(get("-sub_pc_factor_levels", "0").c_str());
    opts_.bjacobi_blocks = std::atoi(get("-pc_bjacobi_blocks", "1").c_str());
  } else {
    std::cerr << " -pc_type " << pc << " is not implemented (none, jacobi, pbjacobi, ilu, lu, bjacobi)" << std::endl;
    return CFDGPU_EINVAL;
  }
  if (options.count("-ksp_gmres_restart")) opts_.restart = std::atoi(options["-ksp_gmres_restart"].c_str());
  if (options.count("-ksp_rtol")) opts_.rtol = std::atof(options["-ksp_rtol"].c_str());
  if (options.count("-ksp_max_it")) opts_.max_it = std::atoi(options["-ksp_max_it"].c_str());
  if (options.count("-ksp_atol")) opts_.atol = std::atof(options["-ksp_atol"].c_str());
  if (options.count("-ksp_divtol")) opts_.dtol = std::atof(options["-ksp_divtol"].c_str());
  if (get("-gpu_precision", "fp64") == "mixed") opts_.precision = CFDGPU_PREC_MIXED;
  if (options.count("-gpu_inner_restart")) opts_.inner_restart = std::atoi(options["-gpu_inner_restart"].c_str());
  if (options.count("-gpu_inner_rtol")) opts_.inner_rtol = std::atof(options["-gpu_inner_rtol"].c_str());
  if (options.count("-gpu_refine_rtol")) opts_.refine_rtol = std::atof(options["-gpu_refine_rtol"].c_str());
  if (options.count("-gpu_refine_atol")) opts_.refine_atol = std::atof(options["-gpu_refine_atol"].c_str());
  if (options.count("-gpu_newton_rtol")) opts_.newton_rtol = std::atof(options["-gpu_newton_rtol"].c_str());
  {
    const std::string f = get("-gpu_formulation", "semi_implicit");
    if (f == "fully_implicit") opts_.formulation = CFDGPU_FORM_FULLY_IMPLICIT;
    else if (f != "semi_implicit") {
      std::cerr << " -gpu_formulation must be semi_implicit or fully_implicit" << std::endl;
      return CFDGPU_EINVAL;
    }
  }

  std::vector<double> xyz((size_t)nNode_global * ndim), dv(nDBC);
  std::vector<int32_t> conn((size_t)nElem_global * npElem), dn(nDBC), dd(nDBC);
  for (int i = 0; i < nNode_global; i++)
    for (int c = 0; c < ndim; c++) xyz[(size_t)i * ndim + c] = node_coords[i][c];
  for (int e = 0; e < nElem_global; e++)
    for (int a = 0; a < npElem; a++) conn[(size_t)e * npElem + a] = elemConn[e][a];
  for (int k = 0; k < nDBC; k++) {
    dn[k] = (int32_t)DirichletBCs[k][0];
    dd[k] = (int32_t)DirichletBCs[k][1];
    dv[k] = DirichletBCs[k][2];
  }
  cfdgpu_mesh m = {ndim, npElem, nNode_global, nElem_global, xyz.data(), conn.data(), nDBC,
                   dn.data(), dd.data(), dv.data()};
  cfdgpu_control c = {elemData[0], elemData[1], {elemData[2], elemData[3], elemData[4]},
                      {elemData[8], elemData[9], elemData[10]}, tis, rhoInf, dt, 1.0e-8, 10};
  const double t0 = now_s();
  deallocatePetscObjects();
  int rc = cfdgpu_create(&m, &c, &opts_, &gpu);
  computerTimePattern = now_s() - t0;
  if (rc != 0) {
    std::cerr << " cfdgpu_create failed: " << cfdgpu_last_error(gpu) << std::endl;
    return rc;
  }
  const std::string guess = get("-gpu_guess", "constant");
  if (guess == "extrapolation") {
    rc = cfdgpu_set_guess_mode(gpu, nullptr, CFDGPU_GUESS_EXTRAPOLATION);
  } else if (guess != "constant") {
    std::cerr << " -gpu_guess must be constant or extrapolation" << std::endl;
    rc = CFDGPU_EINVAL;
  }
  return rc;
}

// Time loop of StabFEM::solveFullyImplicit (src/base/StabFEM2.cpp:593-832)
int StabFEM::solveFullyImplicit()
{
  if (!gpu) return CFDGPU_EINVAL;
  double timeNow = dt, timeFact;
  const double tloop = now_s();
  cfdgpu_step_stats st;
  for (int tstep = 0; tstep < stepsMax; tstep++) {
    if (verbose) {
      printf(" ==================================================================== \n");
      printf(" Time = %f \n", timeNow);
      printf(" ==================================================================== \n");
    }
    timeFact = (timeNow <= 1.0) ? timeNow : 1.0;
    int rc = cfdgpu_step(gpu, timeNow, timeFact, &st);
    if (rc != 0) {
      printf(" PETSc solver not converged. \n\n");
      std::cerr << cfdgpu_last_error(gpu) << std::endl;
      return -1;
    }
    computerTimeAssembly += st.ms_assembly * 1e-3;
    computerTimeSolver += st.ms_solver * 1e-3;
    if (verbose) {
      for (int i = 0; i < st.newton_iters; i++) {
        printf(" Iteration = %d  \t RHS norm = %E \n", i + 1, st.norms[i]);
        if (i < st.newton_iters - (st.converged ? 1 : 0)) printf("\n Convergence in %d iterations.\n\n", st.ksp_its[i]);
      }
    }
    cfdgpu_get_solution(gpu, soln.data());
    if (writeVTU) {
      const double t0 = now_s();
      postProcess();
      computerTimePostprocess += now_s() - t0;
    }
    fout_convdata << timeNow << '\t' << 0.0 << '\t' << 0.0 << std::endl;   // reacVec is never filled
    timeNow = timeNow + dt;
    if (timeNow > timeFinal) break;
  }
  computerTimeTimeLoop = now_s() - tloop;
  return 0;
}

// headless .vtu with the fields of StabFEM::postProcess (src/base/StabFEM3.cpp:6-160)
void StabFEM::postProcess()
{
  char fname[512];
  snprintf(fname, sizeof(fname), "%s-%06d.vtu", infilename.c_str(), fileCount);
  FILE *f = fopen(fname, "w");
  if (!f) return;
  const int ctype = (ndim == 2) ? (npElem == 3 ? 5 : 9) : (npElem == 4 ? 10 : 12);
  fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
  fprintf(f, "<UnstructuredGrid>\n<Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", nNode_global, nElem_global);
  fprintf(f, "<PointData Scalars=\"pressure\" Vectors=\"velocity\">\n<DataArray type=\"Float32\" Name=\"pressure\" format=\"ascii\">\n");
  for (int i = 0; i < nNode_global; i++) fprintf(f, "%.9g ", (float)soln[(size_t)i * ndof + ndim]);
  fprintf(f, "\n</DataArray>\n<DataArray type=\"Float32\" Name=\"procId\" format=\"ascii\">\n");
  for (int i = 0; i < nNode_global; i++) fprintf(f, "0 ");
  fprintf(f, "\n</DataArray>\n<DataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n");
  for (int i = 0; i < nNode_global; i++)
    for (int c = 0; c < 3; c++) fprintf(f, "%.9g ", c < ndim ? (float)soln[(size_t)i * ndof + c] : 0.0f);
  fprintf(f, "\n</DataArray>\n</PointData>\n<CellData Scalars=\"procId\">\n<DataArray type=\"Float32\" Name=\"procId\" format=\"ascii\">\n");
  for (int e = 0; e < nElem_global; e++) fprintf(f, "0 ");
  fprintf(f, "\n</DataArray>\n</CellData>\n<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
  for (int i = 0; i < nNode_global; i++)
    for (int c = 0; c < 3; c++) fprintf(f, "%.9g ", c < ndim ? (float)node_coords[i][c] : 0.0f);
  fprintf(f, "\n</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n");
  for (int e = 0; e < nElem_global; e++)
    for (int a = 0; a < npElem; a++) fprintf(f, "%d ", elemConn[e][a]);
  fprintf(f, "\n</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n");
  for (int e = 0; e < nElem_global; e++) fprintf(f, "%d ", (e + 1) * npElem);
  fprintf(f, "\n</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
  for (int e = 0; e < nElem_global; e++) fprintf(f, "%d ", ctype);
  fprintf(f, "\n</DataArray>\n</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
  fclose(f);
  fileCount++;
}

// src/base/StabFEM.cpp:457-494
int StabFEM::writeResult(std::string &fname)
{
  FILE *f = fopen(fname.c_str(), "w");
  if (!f) {
    std::cout << " Could not open the file in 'StabFEM::writeResult' ... " << std::endl;
    exit(1);
  }
  fprintf(f, "%d\n", nNode_global);
  for (int i = 0; i < nNode_global; i++) {
    for (int c = 0; c < ndof; c++) fprintf(f, c ? "\t%.8f" : "%.8f", soln[(size_t)i * ndof + c]);
    fprintf(f, "\n");
  }
  fclose(f);
  return 0;
}

// src/base/StabFEM.cpp:501-554: 2D nodes must agree within 1e-4 (Euclidean
// over u, v, p); 3D files are read but not compared.
int StabFEM::checkResult(std::string &fname)
{
  std::ifstream in(fname);
  if (in.fail()) {
    std::cout << " Could not open the file in 'StabFEM::checkResult' ... " << std::endl;
    exit(1);
  }
  int nn;
  in >> nn;
  if (nn != nNode_global) return -1;
  if (ndim != 2) return 0;
  for (int i = 0; i < nNode_global; i++) {
    double v[3];
    in >> v[0] >> v[1] >> v[2];
    const size_t k = (size_t)i * ndof;
    v[0] -= soln[k]; v[1] -= soln[k + 1]; v[2] -= soln[k + 2];
    if (std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) > 1.0e-4) return -2;
  }
  return 0;
}

// src/base/StabFEM.cpp:711-727
int StabFEM::printComputerTimes()
{
  printf("\n====================================================================\n");
  printf("\n       Computer time in seconds \n");
  printf("\n====================================================================\n");
  printf("\n\n     (1) Matrix Pattern                  = %12.6f \n", computerTimePattern);
  printf("\n\n     (2) Matrix Assembly                 = %12.6f \n", computerTimeAssembly);
  printf("\n\n     (3) Matrix Solver                   = %12.6f \n", computerTimeSolver);
  printf("\n\n     (4) Post process                    = %12.6f \n", computerTimePostprocess);
  printf("\n\n     (5) Total time in time loop         = %12.6f \n", computerTimeTimeLoop);
  printf("\n\n     (6) Difference (5-2-3-4)            = %12.6f \n",
         computerTimeTimeLoop - computerTimeAssembly - computerTimeSolver - computerTimePostprocess);
  printf("\n\n====================================================================\n\n");
  return 0;
}
