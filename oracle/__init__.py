"""ORACLE -- test infrastructure only (CPU f64 restatement of the reference path)."""
