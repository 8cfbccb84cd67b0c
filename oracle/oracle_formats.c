/*
 * oracle_formats.c — CPU restatement of the reference's format converters
 * (BCSR, DBSR, DASP packing, block statistics).  TEST INFRASTRUCTURE ONLY.
 */
#include "oracle.h"
