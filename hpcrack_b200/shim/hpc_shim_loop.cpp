// Device-resident staggered loop: a drop-in for crack_propagation (crack_propagation.cpp:28-123)
// with the same signature, constants, load schedule, stop test, console lines, F_U.dat format,
// history dumps and VTK output.  u, d and H live on the device for the whole run; each increment
// is one hpc_step call, host copies are made only for the dumps the configuration asks for, and the
// VTK files of d are encoded on the device and written by a host thread while the loop goes on.
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>

#include "crack_propagation.h"
#include "directory_verification.h"
#include "vtk_output.h"
#include "write_read_history.h"
#include "hpc_shim.h"

namespace {
void check(int rc, const char* what) {
  if (rc != HPC_OK) throw std::runtime_error(std::string(what) + ": " + hpc_last_error());
}
}  // namespace

void crack_propagation(Stack* U, const mgdouble& bulK, const mgdouble& G, const mgdouble& gc, MPI_Setting& M,
                       const Parameters& para, const int myid, const int nbprocs) {
  const double small_k = 1.e-5;  // crack_propagation.cpp:32
  const int L = U->maxlevel;
  hpc_ctx* c = hpc_shim_context(U);
  for (int l = 0; l <= L; ++l) {
    check(hpc_upload(c, HPC_BULK, l, 0, &bulK.getLevel(l)[0]), "upload bulK");
    check(hpc_upload(c, HPC_G, l, 0, &G.getLevel(l)[0]), "upload G");
    check(hpc_upload(c, HPC_GC, l, 0, &gc.getLevel(l)[0]), "upload gc");
  }
  std::ofstream F_U("F_U.dat");
  if (F_U.is_open()) {
    if (myid == 0) std::cout << "File opened!" << std::endl;
  } else {
    if (myid == 0) std::cout << "Can not open file!" << std::endl;
    exit(-1);
  }
  if (para.outTdata == 1) folder_verification("Time_step_data");
  griddouble host(bulK.getLevel(L).axis());
  auto fetch = [&](int field, int comp) -> griddouble& {
    check(hpc_download(c, field, L, comp, &host[0]), "download");
    return host;
  };
  hpc_step_params p{};
  p.mg_u = hpc_mg{para.mg_u.nu0, para.mg_u.nu1, para.mg_u.nu2, para.mg_u.gamma, para.mg_u.ncy};
  p.mg_d = hpc_mg{para.mg_d.nu0, para.mg_d.nu1, para.mg_d.nu2, para.mg_d.gamma, para.mg_d.ncy};
  p.small_k = small_k;
  p.lc = para.lc;
  p.voxel_size = para.voxel_size;
  p.ut0 = 0.0;          // Ut0 = Ue (crack_propagation.cpp:71-80)
  p.du_factor = 1.5e-3; // crack_propagation.cpp:76
  p.mech_tol = 1.e-6;   // mechanical_displacement.cpp:88
  p.pf_tol = 1.e-12;    // phase_field.cpp:30-43
  for (int t = 0; t < 5000; t++) {
    if (myid == 0) std::cout << "***** At Time step " << t << std::endl;
    p.t = t;
    double out[8];
    check(hpc_step(c, &p, out), "hpc_step");
    double s6[6];
    check(hpc_get_state(c, s6), "hpc_get_state");
    if (t == 0 && myid == 0) std::cout << "Ue=" << s6[2] << std::endl;
    if (para.outTdata == 1 && (t % para.Tdatafrequence == 0)) {
      write_vector_3D(fetch(HPC_U, 0), "u", myid, t);
      write_vector_3D(fetch(HPC_U, 1), "v", myid, t);
      write_vector_3D(fetch(HPC_U, 2), "w", myid, t);
      write_vector_3D(fetch(HPC_H, 0), "H", myid, t);
      write_vector_3D(fetch(HPC_D, 0), "d", myid, t);
    }
    const double dmax = out[3];
    // write_total_de(U, d, M, "S", "d", "d", L, myid, nbprocs, t) from the device: the same files,
    // written while the next increment runs
    if (t == 0 || dmax >= 0.98) check(hpc_vtk_write(c, "S", HPC_D, L, 1.0, "d", "d", t), "hpc_vtk_write");
    const double Ut = s6[3], delta_U = s6[4], F = out[1];
    if (myid == 0) {
      F_U << "T= " << t << ",U= " << std::setprecision(10) << Ut << " ,Fw= " << std::setprecision(10) << F
          << " ,deltaU= " << delta_U << " ,delatad_max= " << out[2] << std::endl;
    }
    if (F < 0.5) break;
  }
  F_U.close();
  check(hpc_vtk_wait(c), "hpc_vtk_wait");
  hpc_shim_release_all();
}
