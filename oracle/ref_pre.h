/* Forced-include header for the compiled-reference oracle (test infrastructure). */
#ifndef ORACLE_REF_PRE_H
#define ORACLE_REF_PRE_H
extern int oracle_steps;
#endif
