// The opaque handle types of the C ABI (include/stokesdt_b200.h).
#pragma once
#include "engine.h"
#include "lanczos.h"
#include "steric.h"
#include "bd.h"
#include "batch.h"
#include "serve.h"
#include "ewald.h"

struct sdt_spme {
    sdt::SpmeEngine e;
};

struct sdt_lanczos {
    sdt::LanczosState s;
};

struct sdt_steric {
    sdt::StericEngine e;
};

struct sdt_bd {
    sdt::BdState s;
};

struct sdt_batch {
    sdt::BatchState b;
};

struct sdt_serve {
    sdt::ServeState s;
};

struct sdt_ewald {
    sdt::EwaldEngine e;
};
