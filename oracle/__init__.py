"""CPU oracle (test infrastructure): restatement of the reference kernels in C."""
