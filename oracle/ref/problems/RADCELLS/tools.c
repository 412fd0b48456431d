/* No problem-specific tools. */
