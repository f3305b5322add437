/*
 * X-macro list of every member of the structs that cross the drop-in
 * boundary. Expanded twice: by the library (spb_abi_layout_json, offsets of
 * include/sputnipic_ref_layout.h) and by oracle/layout_probe.cpp (offsets of
 * the reference's own headers). The two JSON documents must be equal.
 */
#define SPB_LAYOUT_PARTICLES(X)                                                  \
  X(particles, species_ID) X(particles, npmax) X(particles, nop)                 \
  X(particles, NiterMover) X(particles, n_sub_cycles) X(particles, npcel)        \
  X(particles, npcelx) X(particles, npcely) X(particles, npcelz)                 \
  X(particles, qom) X(particles, u0) X(particles, v0) X(particles, w0)           \
  X(particles, uth) X(particles, vth) X(particles, wth) X(particles, x)          \
  X(particles, y) X(particles, z) X(particles, u) X(particles, v)                \
  X(particles, w) X(particles, q) X(particles, track_particle)

#define SPB_LAYOUT_EMFIELD(X)                                                    \
  X(EMfield, Ex) X(EMfield, Ex_flat) X(EMfield, Ey) X(EMfield, Ey_flat)          \
  X(EMfield, Ez) X(EMfield, Ez_flat) X(EMfield, Bxn) X(EMfield, Bxn_flat)        \
  X(EMfield, Byn) X(EMfield, Byn_flat) X(EMfield, Bzn) X(EMfield, Bzn_flat)

#define SPB_LAYOUT_GRID(X)                                                       \
  X(grid, nxc) X(grid, nxn) X(grid, nyc) X(grid, nyn) X(grid, nzc)               \
  X(grid, nzn) X(grid, dx) X(grid, dy) X(grid, dz) X(grid, invdx)                \
  X(grid, invdy) X(grid, invdz) X(grid, invVOL) X(grid, xStart) X(grid, xEnd)    \
  X(grid, yStart) X(grid, yEnd) X(grid, zStart) X(grid, zEnd) X(grid, Lx)        \
  X(grid, Ly) X(grid, Lz) X(grid, PERIODICX) X(grid, PERIODICY)                  \
  X(grid, PERIODICZ) X(grid, XN_flat) X(grid, XN) X(grid, YN_flat)               \
  X(grid, YN) X(grid, ZN_flat) X(grid, ZN)

#define SPB_LAYOUT_IDS(X)                                                        \
  X(interpDensSpecies, species_ID) X(interpDensSpecies, rhon)                    \
  X(interpDensSpecies, rhon_flat) X(interpDensSpecies, rhoc)                     \
  X(interpDensSpecies, rhoc_flat) X(interpDensSpecies, Jx)                       \
  X(interpDensSpecies, Jx_flat) X(interpDensSpecies, Jy)                         \
  X(interpDensSpecies, Jy_flat) X(interpDensSpecies, Jz)                         \
  X(interpDensSpecies, Jz_flat) X(interpDensSpecies, pxx)                        \
  X(interpDensSpecies, pxx_flat) X(interpDensSpecies, pxy)                       \
  X(interpDensSpecies, pxy_flat) X(interpDensSpecies, pxz)                       \
  X(interpDensSpecies, pxz_flat) X(interpDensSpecies, pyy)                       \
  X(interpDensSpecies, pyy_flat) X(interpDensSpecies, pyz)                       \
  X(interpDensSpecies, pyz_flat) X(interpDensSpecies, pzz)                       \
  X(interpDensSpecies, pzz_flat)

#define SPB_LAYOUT_PARAMETERS(X)                                                 \
  X(parameters, c) X(parameters, fourpi) X(parameters, dt) X(parameters, th)     \
  X(parameters, ncycles) X(parameters, NiterMover) X(parameters, n_sub_cycles)   \
  X(parameters, sort) X(parameters, sort_every_n) X(parameters, sort_cps)        \
  X(parameters, number_of_batches) X(parameters, threads_per_block)              \
  X(parameters, track_particles) X(parameters, n_tracked_particles)              \
  X(parameters, tracking_start_cycle) X(parameters, tracking_end_cycle)          \
  X(parameters, tracking_Lx) X(parameters, tracking_Ly)                          \
  X(parameters, tracking_Lz) X(parameters, tracked_particles_filename)           \
  X(parameters, Lx) X(parameters, Ly) X(parameters, Lz) X(parameters, nxc)       \
  X(parameters, nyc) X(parameters, nzc) X(parameters, x_center)                  \
  X(parameters, y_center) X(parameters, z_center) X(parameters, L_square)        \
  X(parameters, ns) X(parameters, npcelx) X(parameters, npcely)                  \
  X(parameters, npcelz) X(parameters, np) X(parameters, npMax)                   \
  X(parameters, NpMaxNpRatio) X(parameters, qom) X(parameters, rhoINIT)          \
  X(parameters, uth) X(parameters, vth) X(parameters, wth) X(parameters, u0)     \
  X(parameters, v0) X(parameters, w0) X(parameters, PERIODICX)                   \
  X(parameters, PERIODICY) X(parameters, PERIODICZ) X(parameters, PERIODICX_P)   \
  X(parameters, PERIODICY_P) X(parameters, PERIODICZ_P)                          \
  X(parameters, bcPfaceXright) X(parameters, bcPfaceXleft)                       \
  X(parameters, bcPfaceYright) X(parameters, bcPfaceYleft)                       \
  X(parameters, bcPfaceZright) X(parameters, bcPfaceZleft)                       \
  X(parameters, bcPHIfaceXright) X(parameters, bcPHIfaceXleft)                   \
  X(parameters, bcPHIfaceYright) X(parameters, bcPHIfaceYleft)                   \
  X(parameters, bcPHIfaceZright) X(parameters, bcPHIfaceZleft)                   \
  X(parameters, bcEMfaceXright) X(parameters, bcEMfaceXleft)                     \
  X(parameters, bcEMfaceYright) X(parameters, bcEMfaceYleft)                     \
  X(parameters, bcEMfaceZright) X(parameters, bcEMfaceZleft) X(parameters, Vinj) \
  X(parameters, delta) X(parameters, B0x) X(parameters, B0y) X(parameters, B0z)  \
  X(parameters, Nwaves) X(parameters, dBoB0) X(parameters, pitch_angle)          \
  X(parameters, energy) X(parameters, SmoothON) X(parameters, SmoothValue)       \
  X(parameters, SmoothTimes) X(parameters, verbose) X(parameters, RESTART)       \
  X(parameters, PoissonCorrection) X(parameters, CGtol) X(parameters, GMREStol)  \
  X(parameters, first_cycle_n) X(parameters, FieldOutputCycle)                   \
  X(parameters, ParticlesOutputCycle) X(parameters, RestartOutputCycle)          \
  X(parameters, DiagnosticsOutputCycle) X(parameters, inputfile)                 \
  X(parameters, SaveDirName) X(parameters, RestartDirName) X(parameters, WaveFile)

#define SPB_LAYOUT_IDN(X)                                                        \
  X(interpDensNet, rhon) X(interpDensNet, rhon_flat) X(interpDensNet, rhoc)      \
  X(interpDensNet, rhoc_flat) X(interpDensNet, Jx) X(interpDensNet, Jx_flat)     \
  X(interpDensNet, Jy) X(interpDensNet, Jy_flat) X(interpDensNet, Jz)            \
  X(interpDensNet, Jz_flat) X(interpDensNet, pxx) X(interpDensNet, pxx_flat)     \
  X(interpDensNet, pxy) X(interpDensNet, pxy_flat) X(interpDensNet, pxz)         \
  X(interpDensNet, pxz_flat) X(interpDensNet, pyy) X(interpDensNet, pyy_flat)    \
  X(interpDensNet, pyz) X(interpDensNet, pyz_flat) X(interpDensNet, pzz)         \
  X(interpDensNet, pzz_flat)

#define SPB_LAYOUT_AUX(X)                                                        \
  X(interpDens_aux, rhoh) X(interpDens_aux, Jxh) X(interpDens_aux, Jyh)          \
  X(interpDens_aux, Jzh)

#define SPB_LAYOUT_ALL(X)                                                        \
  SPB_LAYOUT_PARTICLES(X) SPB_LAYOUT_EMFIELD(X) SPB_LAYOUT_GRID(X)               \
  SPB_LAYOUT_IDS(X) SPB_LAYOUT_IDN(X) SPB_LAYOUT_AUX(X) SPB_LAYOUT_PARAMETERS(X)

#define SPB_LAYOUT_STRUCTS(S)                                                    \
  S(particles) S(EMfield) S(grid) S(interpDensSpecies) S(interpDensNet)          \
  S(interpDens_aux) S(parameters)

/* Appends `"struct.member": offset,` pairs and `"struct": sizeof` to a
 * std::string; used by both expansions. */
#define SPB_LAYOUT_EMIT_MEMBER(st, mb)                                           \
  out += "\"" #st "." #mb "\": " + std::to_string(offsetof(st, mb)) + ",\n";
#define SPB_LAYOUT_EMIT_SIZE(st)                                                 \
  out += "\"sizeof " #st "\": " + std::to_string(sizeof(st)) + ",\n";
