// Temporary definitions of entry points that are not implemented yet.
#include "jxb.h"
extern "C" int jxb_synapse_forward(const JxbSynArgs*, void*) { return JXB_ERR_ARG; }
extern "C" int jxb_synapse_backward(const JxbSynArgs*, void*) { return JXB_ERR_ARG; }
extern "C" int jxb_tree_solve_levels(int, const void*, const void*, const void*, const void*, void*, int64_t, const JxbTreeSchedule*, void*) { return JXB_ERR_ARG; }
extern "C" int jxb_tree_solve_registers(int, const void*, const void*, const void*, const void*, void*, int64_t, const JxbRegSchedule*, void*) { return JXB_ERR_ARG; }
