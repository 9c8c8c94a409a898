# Parameterises the compile-time constants of PIC/3d_pic458_domain.c (lines
# 54-103 and init_grid's damping amplitude at :295) so that one recipe can build
# the reference at any test geometry. Values come from -D flags on the compile line.
# The substitutions touch #define values only; no statement of the reference changes.
s|^#define me (mi/100.)//.*|#define me (mi/ORACLE_MASS_RATIO)|
s|^#define dx 1\.5//5\.$|#define dx ORACLE_DX|
s|^#define dt 1\.5E-9//5\.E-9$|#define dt ORACLE_DT|
s|^#define Grid_Nx 4 .*|#define Grid_Nx ORACLE_NX|
s|^#define Grid_Ny 4 .*|#define Grid_Ny ORACLE_NY|
s|^#define Grid_Nz 512 .*|#define Grid_Nz ORACLE_NZ|
s|^#define Np 16$|#define Np ORACLE_NP|
s|^#define V 1\.2E7 .*|#define V ORACLE_V|
s|^#define Nall 5E10 .*|#define Nall ORACLE_NALL|
s|^#define Ti 1e9 .*|#define Ti ORACLE_TI|
s|^#define Te 1e9$|#define Te ORACLE_TE|
s|^#define R 2\.//=4\.\*dx$|#define R ORACLE_R|
s|^#define I 6\.8e7 .*|#define I ORACLE_I|
s|^#define alpha (Pi/2\.)$|#define alpha ORACLE_ALPHA|
s|^#define Step 300001$|#define Step oracle_steps|
s|^#define Absorb_grid 32 .*|#define Absorb_grid ORACLE_ABSORB|
s|^#define Absorb_grid2 40 .*|#define Absorb_grid2 ORACLE_ABSORB2|
s|^#define THREAD_N 4$|#define THREAD_N ORACLE_THREADS|
s|^int active_thread=1;$|int active_thread=ORACLE_ACTIVE_THREADS;|
s|^#define PROCESS_Nx 128$|#define PROCESS_Nx ORACLE_PNX|
s|^#define PROCESS_Ny 128$|#define PROCESS_Ny ORACLE_PNY|
s|^#define PACK_N 80000$|#define PACK_N ORACLE_PACK_N|
s|^  const double a=1e-6;$|  const double a=ORACLE_SIGMA_A;|
s|^#define Absorb_grid3 40  //particle$|#define Absorb_grid3 ORACLE_ABSORB3|
s|^#define PHI(x) $|#if ORACLE_PHI\n#define PHI(...) __VA_ARGS__\n#else\n#define PHI(...)\n#endif|
