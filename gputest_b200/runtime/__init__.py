"""Running many cases: ``run_batch`` (mesh-file jobs solved as block-diagonal device batches)."""
