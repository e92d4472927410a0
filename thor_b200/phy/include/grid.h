// The reference's grid header; a module reads the grid through ESP's members (esp.h).
#pragma once
