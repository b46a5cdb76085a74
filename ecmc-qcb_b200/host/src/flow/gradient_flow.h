// flow/gradient_flow.h -- Wilson flow state (reference src/flow/gradient_flow.h:11-27) on the GPU:
// fused RK3 stages over device-resident buffers; field_c views the flowed field.
#pragma once
#include <memory>

#include "../gauge/GaugeField.h"
#include "../mpi/MpiTopology.h"

class GradientFlow {
   public:
    double epsilon;

   private:
    qcb_flow fl_ = nullptr;
    std::unique_ptr<GaugeField> holder_;

   public:
    GaugeField& field_c;
    const GeometryCB* geo_p;

    explicit GradientFlow(double epsilon_, const GaugeField& field, const GeometryCB& geo);
    GradientFlow(const GradientFlow&) = delete;
    GradientFlow& operator=(const GradientFlow&) = delete;
    ~GradientFlow();
    void copy(const GaugeField& field);
    void rk3_step(mpi::MpiTopology& topo);
    // The reference's separate passes (gradient_flow.cpp:17-121); force_0 and force_1 live on the
    // device inside the flow state (the reference's public force_0 / force_1 fields are not exposed).
    void compute_force(int i);
    void compute_w1();
    void compute_w2();
    void replace_force_0();
    void compute_w3();
    qcb_flow handle() const { return fl_; }

   private:
    void run_pass(int pass, const char* what);

   public:
};
