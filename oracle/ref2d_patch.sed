# Parameterises the compile-time constants of PIC2D/2d_pic278_mpi.c (lines
# 31-87 and init_grid's damping amplitude at :228) so that one recipe can build
# the 2D reference at any test geometry, at MPI size 1 (PROCESS_N = 1). Values
# come from -D flags on the compile line. Only #define values and the damping
# amplitude change; no statement of the reference changes.
s|^#define q GSL_CONST_MKSA_ELECTRON_CHARGE$|#define q ORACLE_Q|
s|^#define mi GSL_CONST_MKSA_MASS_PROTON$|#define mi ORACLE_MI|
s|^#define me GSL_CONST_MKSA_MASS_ELECTRON //.*|#define me ORACLE_ME|
s|^#define mu0 GSL_CONST_MKSA_VACUUM_PERMEABILITY$|#define mu0 ORACLE_MU0|
s|^#define e0 GSL_CONST_MKSA_VACUUM_PERMITTIVITY$|#define e0 ORACLE_E0|
s|^#define kb GSL_CONST_MKSA_BOLTZMANN$|#define kb ORACLE_KB|
s|^#define C 3\.0E8$|#define C ORACLE_C|
s|^#define R 75\.0//.*|#define R ORACLE_R|
s|^#define I 4\.0E3 //.*|#define I ORACLE_I|
s|^#define alpha 0\. //.*|#define alpha ORACLE_ALPHA|
s|^#define dx 30\. //.*|#define dx ORACLE_DX|
s|^#define dtf 0\.6E-7$|#define dtf ORACLE_DT|
s|^#define dti (0\.6E-7)//0\.6E-7$|#define dti (ORACLE_DT)|
s|^#define dte (0\.6E-7)$|#define dte (ORACLE_DT)|
s|^#define Grid_Nx 16 //.*|#define Grid_Nx ORACLE_NX|
s|^#define Grid_Nz 512 //.*|#define Grid_Nz ORACLE_NZ|
s|^#define Np 4$|#define Np ORACLE_NP|
s|^#define V 5\.0E5  //.*|#define V ORACLE_V|
s|^#define Nall 5\.0E6 //.*|#define Nall ORACLE_NALL|
s|^#define Ti 1\.0E6$|#define Ti ORACLE_TI|
s|^#define Te 1\.0E6$|#define Te ORACLE_TE|
s|^#define PACK_N 40000$|#define PACK_N ORACLE_PACK_N|
s|^#define Step 10000001$|#define Step oracle_steps|
s|^#define Absorb_grid 32  //field$|#define Absorb_grid ORACLE_ABSORB|
s|^#define Absorb_grid2 16  //particle$|#define Absorb_grid2 ORACLE_ABSORB2|
s|^#define Absorb_grid3 32 //phi$|#define Absorb_grid3 ORACLE_ABSORB3|
s|^#define THREAD_N 2$|#define THREAD_N 1|
s|^#define PROCESS_N 32$|#define PROCESS_N 1|
s|^  const double a=1E-9;$|  const double a=ORACLE_SIGMA_A;|
