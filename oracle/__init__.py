"""CPU oracle of the B200 BEM path (test infrastructure only; see bem3d_oracle.h)."""
