/* Forced-include header for the compiled-reference oracle (test infrastructure). */
#ifndef ORACLE_REF_PRE_H
#define ORACLE_REF_PRE_H
extern int oracle_steps;
/* active_thread (:110): OpenMP threads of fdtd's particle loops; 1 as shipped */
#ifndef ORACLE_ACTIVE_THREADS
#define ORACLE_ACTIVE_THREADS 1
#endif
#endif
