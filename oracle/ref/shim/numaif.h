/* Empty stand-in: the compiled-reference build never calls libnuma. */
