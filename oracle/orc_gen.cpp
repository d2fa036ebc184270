// ORACLE — test infrastructure only.  The workload input generators and the
// reference parameter defaults (zebraflow_b200/csrc/zf_gen.cpp, plain host C++)
// compiled into the CPU arm's library under the orc_ prefix, so that a CPU run
// builds exactly the inputs the GPU library would without loading it.
#define ZF_SYM(name) orc_##name
#include "../zebraflow_b200/csrc/zf_gen.cpp"
