"""B200 adding-doubling radiative-transfer engine."""
