// Part of the ParlayLib-API shim (test infrastructure for the oracle only).
#pragma once
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>
#include "shim_core.h"
