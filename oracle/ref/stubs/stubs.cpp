/* Abort-stubs for the METIS / SCOTCH entry points the reference links
 * against.  Reaching one means a test asked the compiled reference for a
 * partition or ordering, which this build cannot provide. */
#include <cstdio>
#include <cstdlib>
#include "metis.h"
#include "scotch.h"

static void unavailable(const char *what) {
  std::fprintf(stderr, "oracle/_ref: %s is not available in this build\n", what);
  std::abort();
}
extern "C" {
int METIS_SetDefaultOptions(idx_t *) { unavailable("METIS"); return 0; }
int METIS_PartGraphKway(idx_t *, idx_t *, idx_t *, idx_t *, idx_t *, idx_t *,
                        idx_t *, idx_t *, real_t *, real_t *, idx_t *, idx_t *,
                        idx_t *) { unavailable("METIS"); return 0; }
int SCOTCH_graphInit(SCOTCH_Graph *) { unavailable("SCOTCH"); return 0; }
void SCOTCH_graphExit(SCOTCH_Graph *) {}
int SCOTCH_graphBuild(SCOTCH_Graph *, SCOTCH_Num, SCOTCH_Num, const SCOTCH_Num *,
                      const SCOTCH_Num *, const SCOTCH_Num *, const SCOTCH_Num *,
                      SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *) {
  unavailable("SCOTCH"); return 0;
}
int SCOTCH_graphCheck(const SCOTCH_Graph *) { unavailable("SCOTCH"); return 0; }
int SCOTCH_stratInit(SCOTCH_Strat *) { unavailable("SCOTCH"); return 0; }
void SCOTCH_stratExit(SCOTCH_Strat *) {}
int SCOTCH_stratGraphOrder(SCOTCH_Strat *, const char *) { unavailable("SCOTCH"); return 0; }
int SCOTCH_graphOrder(SCOTCH_Graph *, SCOTCH_Strat *, SCOTCH_Num *, SCOTCH_Num *,
                      SCOTCH_Num *, SCOTCH_Num *, SCOTCH_Num *) {
  unavailable("SCOTCH"); return 0;
}
}
