"""CPU oracle (test infrastructure only; see ``hf_oracle``)."""
