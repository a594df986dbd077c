"""The oracle: a CPU restatement of the engine's WGSL march (test infrastructure only)."""
