// Internal host-side helpers of the firtez-dz B200 library.
#pragma once
#include <vector>

#include "../../include/fz_b200.h"

int fzh_lines_parse(const char* text, fz_line* out, int maxn);
int fzh_zeeman(const fz_line& ln, std::vector<double>& shift, std::vector<double>& strength, std::vector<int>& type);
