/* Periodic in every direction: no problem-specific boundary condition. */
