"""FP64 CPU restatement of wavecore's step: the parity checker and CPU baseline (test infrastructure only)."""
