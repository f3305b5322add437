/*
 * Layout-compatible declarations of the sputniPIC structs that cross the
 * mover / P2G boundary, for callers that do not compile against the
 * reference's own headers (FFI users, and this library's own build).
 *
 * The field order, types and padding must equal the reference's, because the
 * structs ARE the interface: a maintainer swaps src/Mover.cpp for this
 * library and the unchanged reference driver passes its own structs in.
 * tests/test_abi_cpu.py checks every offset below against offsets measured
 * from the reference headers (tests/golden/abi_layout.json).
 *
 *   struct particles          include/Particles.h:11-56
 *   struct EMfield            include/EMfield.h:8-25
 *   struct grid               include/Grid.h:11-63
 *   struct interpDensSpecies  include/InterpDensSpecies.h:9-40
 *   struct interpDensNet      include/InterpDensNet.h:9-39
 *   struct parameters         include/Parameters.h:10-235
 *
 * Precision: the reference's default PrecisionTypes (include/PrecisionTypes.h:
 * 6-10), i.e. FPpart = FPfield = FPinterp = float.
 *
 * Do not include this header together with the reference's headers: the
 * reference's own definitions are the same structs.
 */
#ifndef SPUTNIPIC_REF_LAYOUT_H
#define SPUTNIPIC_REF_LAYOUT_H

#ifdef __cplusplus
#include <string>
#else
#include <stdbool.h>
#include <stddef.h>
#endif

typedef float spb_FPpart;
typedef float spb_FPfield;
typedef float spb_FPinterp;

#define SPB_NS_MAX 6 /* NS_MAX, include/Parameters.h:7 */

#ifdef __cplusplus
typedef std::string spb_string;
#else
/* Storage of a 64-bit libstdc++ std::string (pointer, size, 16-byte union).
 * C callers never touch it; the library never reads it. */
typedef struct spb_string {
  void *p_;
  size_t n_;
  char buf_[16];
} spb_string;
#endif

struct particles {
  int species_ID;
  long npmax;
  long nop;
  int NiterMover;
  int n_sub_cycles;
  int npcel;
  int npcelx;
  int npcely;
  int npcelz;
  spb_FPpart qom;
  spb_FPpart u0, v0, w0;
  spb_FPpart uth, vth, wth;
  spb_FPpart *x;
  spb_FPpart *y;
  spb_FPpart *z;
  spb_FPpart *u;
  spb_FPpart *v;
  spb_FPpart *w;
  spb_FPinterp *q;
  bool *track_particle;
};

struct EMfield {
  spb_FPfield ***Ex;
  spb_FPfield *Ex_flat;
  spb_FPfield ***Ey;
  spb_FPfield *Ey_flat;
  spb_FPfield ***Ez;
  spb_FPfield *Ez_flat;
  spb_FPfield ***Bxn;
  spb_FPfield *Bxn_flat;
  spb_FPfield ***Byn;
  spb_FPfield *Byn_flat;
  spb_FPfield ***Bzn;
  spb_FPfield *Bzn_flat;
};

struct grid {
  int nxc;
  int nxn;
  int nyc;
  int nyn;
  int nzc;
  int nzn;
  double dx;
  double dy;
  double dz;
  spb_FPfield invdx;
  spb_FPfield invdy;
  spb_FPfield invdz;
  spb_FPfield invVOL;
  double xStart, xEnd, yStart, yEnd, zStart, zEnd;
  double Lx, Ly, Lz;
  bool PERIODICX;
  bool PERIODICY;
  bool PERIODICZ;
  spb_FPfield *XN_flat;
  spb_FPfield ***XN;
  spb_FPfield *YN_flat;
  spb_FPfield ***YN;
  spb_FPfield *ZN_flat;
  spb_FPfield ***ZN;
};

struct interpDensSpecies {
  int species_ID;
  spb_FPinterp ***rhon;
  spb_FPinterp *rhon_flat;
  spb_FPinterp ***rhoc;
  spb_FPinterp *rhoc_flat;
  spb_FPinterp ***Jx;
  spb_FPinterp *Jx_flat;
  spb_FPinterp ***Jy;
  spb_FPinterp *Jy_flat;
  spb_FPinterp ***Jz;
  spb_FPinterp *Jz_flat;
  spb_FPinterp ***pxx;
  spb_FPinterp *pxx_flat;
  spb_FPinterp ***pxy;
  spb_FPinterp *pxy_flat;
  spb_FPinterp ***pxz;
  spb_FPinterp *pxz_flat;
  spb_FPinterp ***pyy;
  spb_FPinterp *pyy_flat;
  spb_FPinterp ***pyz;
  spb_FPinterp *pyz_flat;
  spb_FPinterp ***pzz;
  spb_FPinterp *pzz_flat;
};

/* Net densities, the sum over species (include/InterpDensNet.h). */
struct interpDensNet {
  spb_FPinterp ***rhon;
  spb_FPinterp *rhon_flat;
  spb_FPinterp ***rhoc;
  spb_FPinterp *rhoc_flat;
  spb_FPinterp ***Jx;
  spb_FPinterp *Jx_flat;
  spb_FPinterp ***Jy;
  spb_FPinterp *Jy_flat;
  spb_FPinterp ***Jz;
  spb_FPinterp *Jz_flat;
  spb_FPinterp ***pxx;
  spb_FPinterp *pxx_flat;
  spb_FPinterp ***pxy;
  spb_FPinterp *pxy_flat;
  spb_FPinterp ***pxz;
  spb_FPinterp *pxz_flat;
  spb_FPinterp ***pyy;
  spb_FPinterp *pyy_flat;
  spb_FPinterp ***pyz;
  spb_FPinterp *pyz_flat;
  spb_FPinterp ***pzz;
  spb_FPinterp *pzz_flat;
};

/* Implicit-source densities of the field solver (include/InterpDens_aux.h:
 * 6-13): rho hat on the cell centres, J hat on the nodes, each a 3-level
 * pointer over one contiguous block (newArr3). */
struct interpDens_aux {
  spb_FPinterp ***rhoh;
  spb_FPinterp ***Jxh;
  spb_FPinterp ***Jyh;
  spb_FPinterp ***Jzh;
};

struct parameters {
  double c;
  double fourpi;
  double dt;
  double th;
  int ncycles;
  int NiterMover;
  int n_sub_cycles;
  bool sort;
  long sort_every_n;
  long sort_cps;
  int number_of_batches;
  long threads_per_block;
  bool track_particles;
  long n_tracked_particles;
  long tracking_start_cycle;
  long tracking_end_cycle;
  long tracking_Lx;
  long tracking_Ly;
  long tracking_Lz;
  spb_string tracked_particles_filename;
  double Lx;
  double Ly;
  double Lz;
  int nxc;
  int nyc;
  int nzc;
  double x_center;
  double y_center;
  double z_center;
  double L_square;
  int ns;
  int npcelx[SPB_NS_MAX];
  int npcely[SPB_NS_MAX];
  int npcelz[SPB_NS_MAX];
  long np[SPB_NS_MAX];
  long npMax[SPB_NS_MAX];
  double NpMaxNpRatio;
  double qom[SPB_NS_MAX];
  double rhoINIT[SPB_NS_MAX];
  double uth[SPB_NS_MAX];
  double vth[SPB_NS_MAX];
  double wth[SPB_NS_MAX];
  double u0[SPB_NS_MAX];
  double v0[SPB_NS_MAX];
  double w0[SPB_NS_MAX];
  bool PERIODICX;
  bool PERIODICY;
  bool PERIODICZ;
  bool PERIODICX_P;
  bool PERIODICY_P;
  bool PERIODICZ_P;
  int bcPfaceXright;
  int bcPfaceXleft;
  int bcPfaceYright;
  int bcPfaceYleft;
  int bcPfaceZright;
  int bcPfaceZleft;
  int bcPHIfaceXright;
  int bcPHIfaceXleft;
  int bcPHIfaceYright;
  int bcPHIfaceYleft;
  int bcPHIfaceZright;
  int bcPHIfaceZleft;
  int bcEMfaceXright;
  int bcEMfaceXleft;
  int bcEMfaceYright;
  int bcEMfaceYleft;
  int bcEMfaceZright;
  int bcEMfaceZleft;
  double Vinj;
  double delta;
  double B0x;
  double B0y;
  double B0z;
  int Nwaves;
  double dBoB0;
  double pitch_angle;
  double energy;
  bool SmoothON;
  double SmoothValue;
  int SmoothTimes;
  bool verbose;
  bool RESTART;
  bool PoissonCorrection;
  double CGtol;
  double GMREStol;
  int first_cycle_n;
  int FieldOutputCycle;
  int ParticlesOutputCycle;
  int RestartOutputCycle;
  int DiagnosticsOutputCycle;
  spb_string inputfile;
  spb_string SaveDirName;
  spb_string RestartDirName;
  spb_string WaveFile;
};

#endif /* SPUTNIPIC_REF_LAYOUT_H */
