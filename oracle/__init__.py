"""ORACLE — test infrastructure only: CPU restatement of polysolve's MAS-PCG (parity unpinned)."""
