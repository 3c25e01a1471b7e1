// Stand-in for a header that algorithms/utils/rangeSearch.h includes but the
// reference checkout does not contain. Nothing from it is used by the range
// search code this oracle compiles, so it is empty.
#pragma once
