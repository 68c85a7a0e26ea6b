/* Declarations standing in for SCOTCH's scotch.h, enough for the reference's
 * reorder.hpp to compile.  The serial loop never calls SCOTCH; the definitions
 * in stubs.cpp abort if reached. */
#ifndef FOT_STUB_SCOTCH_H
#define FOT_STUB_SCOTCH_H
#include <stdint.h>
typedef int32_t SCOTCH_Num;
typedef struct { double dummy[16]; } SCOTCH_Graph;
typedef struct { double dummy[4]; } SCOTCH_Strat;
#ifdef __cplusplus
extern "C" {
#endif
int SCOTCH_graphInit(SCOTCH_Graph *);
void SCOTCH_graphExit(SCOTCH_Graph *);
int SCOTCH_graphBuild(SCOTCH_Graph *, SCOTCH_Num, SCOTCH_Num, const SCOTCH_Num *,
                      const SCOTCH_Num *, const SCOTCH_Num *, const SCOTCH_Num *,
                      SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *);
int SCOTCH_graphCheck(const SCOTCH_Graph *);
int SCOTCH_stratInit(SCOTCH_Strat *);
void SCOTCH_stratExit(SCOTCH_Strat *);
int SCOTCH_stratGraphOrder(SCOTCH_Strat *, const char *);
int SCOTCH_graphOrder(SCOTCH_Graph *, SCOTCH_Strat *, SCOTCH_Num *, SCOTCH_Num *,
                      SCOTCH_Num *, SCOTCH_Num *, SCOTCH_Num *);
#ifdef __cplusplus
}
#endif
#endif
