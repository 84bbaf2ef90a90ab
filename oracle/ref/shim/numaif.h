/* Empty stand-in: the checker build never calls libnuma. */
