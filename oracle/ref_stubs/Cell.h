// The one member of the reference's Cell that dc_backend.cpp reads. TEST INFRASTRUCTURE ONLY.
#pragma once
class Cell {
public:
    bool has_vertex = false;
};
