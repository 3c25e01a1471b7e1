// Part of the ParlayLib-API shim (test infrastructure for the oracle only).
#pragma once
#include <random>
#include "internal/shim_core.h"
