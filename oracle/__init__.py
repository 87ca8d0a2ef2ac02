"""ORACLE — test infrastructure (the CPU restatement used as the parity checker)."""
