/* Empty configure result: the emulator builds the reference sources with
 * every optional feature (debug checks, logging, PSHMEM) switched off. */
