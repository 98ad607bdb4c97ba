"""Drop-in counterparts of the reference package of the same name."""
