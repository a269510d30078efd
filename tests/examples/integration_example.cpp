// Integration example for C++ hosts that drove the reference's engine class
// in process: the mirror of include/ldp_engine.hpp.  Compiled by
// tests/test_integration_examples_cpu.py.
#include "ldp_engine.hpp"
int examples(ldp_ctx* ctx, ldp_params p) {
ldp::LangevinEquationSIMDMultiple engine(ctx, p, /*lanes*/ 8, /*ranks*/ 4, /*rank*/ 0);
engine.Initialize(1234);
for (int trial = 0; trial < p.number_of_runs; ++trial) {
    if (!engine.Integrate(trial)) return 1;          /* error printed on stderr */
    double mfpt = engine.GetFirstPassageTimeAverage(0);   /* lane 0 of this trial */
    double first = engine.GetFirstPassageTime(0, 0);      /* its first event (FP64 plain) */
    double steps_in_state1 = engine.GetStateCount(0, 1);
    if (p.write_restart && !engine.WriteRestartFile(trial)) return 1;
}
return 0;
}
