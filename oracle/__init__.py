"""Oracle package: test infrastructure only (see ``jla_oracle.c``)."""
