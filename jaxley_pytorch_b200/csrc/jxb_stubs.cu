// Temporary definitions of entry points that are not implemented yet.
#include "jxb.h"
extern "C" int jxb_synapse_forward(const JxbSynArgs*, void*) { return JXB_ERR_ARG; }
extern "C" int jxb_synapse_backward(const JxbSynArgs*, void*) { return JXB_ERR_ARG; }
