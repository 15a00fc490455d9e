"""B200-native boundary-element hot path of NeuralAT (Helmholtz BEM on triangle meshes).

``neuralat_b200.bem`` mirrors the reference's ``src/bem`` Python API; the
numerical work runs in ``libbemb200.so`` (hand-written sm_100a CUDA, C ABI in
``include/bem_b200.h``).
"""
__version__ = "0.1.0"
