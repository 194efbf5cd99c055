# Stream edit of C/eduPIC.cc for the reference CPU build (see Makefile).
# 1. simulation parameters (C/eduPIC.cc:49-58) and particle capacity (:89)
#    become macros; edupic_hooks.h defaults them to the original values.
s/^\(const int  *N_G  *= *\)400;/\1EDUPIC_N_G;/
s/^\(const int  *N_T  *= *\)4000;/\1EDUPIC_N_T;/
s/^\(const double  *VOLTAGE  *= *\)250\.0;/\1EDUPIC_VOLTAGE;/
s/^\(const double  *L  *= *\)0\.025;/\1EDUPIC_L;/
s/^\(const double  *PRESSURE  *= *\)10\.0;/\1EDUPIC_PRESSURE;/
s/^\(const double  *WEIGHT  *= *\)7\.0e4;/\1EDUPIC_WEIGHT;/
s/^\(const int  *N_INIT  *= *\)1000;/\1EDUPIC_N_INIT;/
s/^\(const int  *MAX_N_P = *\)1000000;/\1EDUPIC_MAX_N_P;/
# 2. fixed seed instead of std::random_device (C/eduPIC.cc:165)
s/^std::mt19937 MTgen(rd());/std::mt19937 MTgen(EDUPIC_SEED);/
# 3. a bounded number of steps per call and a counting hook at the top of
#    every time step (C/eduPIC.cc:514-515)
s/for (t=0; t<N_T; t++){/for (t=0; t<EDUPIC_STEPS_PER_CYCLE; t++){/
s|Time += DT_E;  *// update of the total simulated time|Time += DT_E; EDUPIC_STEP_HOOK(t);|
