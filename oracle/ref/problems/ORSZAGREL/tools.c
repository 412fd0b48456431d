/* No problem-specific helper routines. */
