"""CPU oracle package (test infrastructure only): a restatement of the
reference INS2D MATLAB algorithm used as the checker and CPU baseline."""
